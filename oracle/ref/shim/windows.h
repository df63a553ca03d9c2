/*
 * Linux stand-in for <windows.h> as seen by the reference INT3 engine.
 *
 * TEST INFRASTRUCTURE ONLY: this header lets the reference CPU sources
 * (cfms_tomo/Tomo_Shell_vc_src/cpu_src/*.cpp) compile unmodified with g++ so
 * they can serve as the parity oracle and as the timed CPU baseline.  It is
 * never linked into the product library.
 *
 * The reference reaches <windows.h> through pch.h -> framework.h
 * (cfms_tomo/Tomo_Shell_vc_src/framework.h:5) and uses only three things
 * from the Win32 / MSVC CRT world:
 *   - _dupenv_s  (debug env switches, e.g. STomoSh_INT3.cpp:23, Tomo_Shell2026.cpp:145,163)
 *   - fopen_s    (debug CSV dumps, e.g. STomoSh_INT3.cpp:92)
 *   - the min/max function-like macros windows.h defines without NOMINMAX
 *     (STomoSh_INT3.cpp:560,1344,1346,1359,1403,1404)
 * All three are arithmetic-neutral.  min/max are provided as templates with
 * the same selection rule as the Win32 macros so that <algorithm> still
 * compiles.
 *
 * The reference also calls ::sqrt, ::sin and pow without including any math
 * header in several units (Tomo_types.cpp:182,194, STomoSh_INT3.cpp:756,1328,
 * STomoVolMassInfo.cpp:383); under MSVC the CRT/STL headers make the C++
 * math overloads visible in the global namespace.  The C++ <math.h> wrapper
 * does the same under libstdc++, so float arguments select the float
 * overloads (sinf, sqrtf, powf) in every reference unit, exactly as in
 * SMatrix4f.cpp which includes <math.h> itself.
 */
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <math.h>

typedef int errno_t;

/* Win32 _dupenv_s: malloc'd copy of an environment variable, NULL if unset. */
static inline errno_t _dupenv_s(char** buf, size_t* len, const char* name)
{
  if (buf == nullptr) return 22;
  *buf = nullptr;
  if (len != nullptr) *len = 0;
  const char* v = std::getenv(name);
  if (v == nullptr) return 0;
  size_t n = std::strlen(v) + 1;
  char* copy = static_cast<char*>(std::malloc(n));
  if (copy == nullptr) return 12;
  std::memcpy(copy, v, n);
  *buf = copy;
  if (len != nullptr) *len = n;
  return 0;
}

/* Win32 fopen_s: the reference builds "%s\\name.csv" paths; only used by
 * env-gated debug dumps that the oracle never enables. */
static inline errno_t fopen_s(FILE** fp, const char* name, const char* mode)
{
  if (fp == nullptr) return 22;
  *fp = std::fopen(name, mode);
  return (*fp == nullptr) ? 2 : 0;
}

/* windows.h: #define max(a,b) (((a) > (b)) ? (a) : (b)), min likewise. */
template <class T> static inline T max(T a, T b) { return (a > b) ? a : b; }
template <class T> static inline T min(T a, T b) { return (a < b) ? a : b; }
