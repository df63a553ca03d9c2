// Row spans of a triangle's pixel box: per column, the rows whose pixel
// centres can pass the pre-reject of the barycentric test.  Every pixel the
// exact test accepts passes the pre-reject, so a box whose spans are all
// empty holds no accepted pixel, and a search for one may skip every pixel
// outside the spans.  The binning kernel uses this for the "does any pixel
// of the box hit" test of strip-spanning triangles.
//
// The pre-reject compares the sign-adjusted barycentric numerators
//   vs = s * (d11 * d20 - d01 * d21),  ws = s * (d00 * d21 - d01 * d20),
//   d20 = e2x * e0x + e2y * e0y,       d21 = e2x * e1x + e2y * e1y,
// evaluated in float, with vs >= rlo, ws >= rlo, vs + ws <= ruhi (and upper
// bounds on vs and ws alone, which a span may ignore: it may be longer than
// needed, never shorter).  For a fixed column (fixed float e2x) both are
// linear in e2y, so each bound is a half-line in e2y; span_setup and
// span_rows compute those half-lines in float with a rigorous bound on every
// rounding, stated where it is used.
//
// Everything here is plain IEEE float arithmetic (and directed roundings),
// so the same code compiles for the host, where a test checks the spans
// against the float pre-reject on random triangles.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define TOMO_HD __host__ __device__ __forceinline__
#else
#define TOMO_HD inline
#endif

namespace tomo {

// Directed float subtraction / addition (device: one instruction; host: the
// exact double result rounded outward, which is the same value).
TOMO_HD float sub_down(float a, float b)
{
#ifdef __CUDA_ARCH__
  return __fsub_rd(a, b);
#else
  const double d = (double)a - (double)b;
  float f = (float)d;
  if ((double)f > d) f = nextafterf(f, -INFINITY);
  return f;
#endif
}
TOMO_HD float add_up(float a, float b)
{
#ifdef __CUDA_ARCH__
  return __fadd_ru(a, b);
#else
  const double d = (double)a + (double)b;
  float f = (float)d;
  if ((double)f < d) f = nextafterf(f, INFINITY);
  return f;
#endif
}
// IEEE reciprocal, round to nearest (device: __frcp_rn; host: 1 / x).
TOMO_HD float recip_rn(float x)
{
#ifdef __CUDA_ARCH__
  return __frcp_rn(x);
#else
  return 1.0f / x;
#endif
}

// Per-triangle constants of the span computation.  Only the three one-sided
// bounds that shape the region are used (vs >= rlo, ws >= rlo,
// vs + ws <= ruhi); the upper bounds of vs and ws alone would only shorten
// spans further, and a span may be longer than needed.
struct SpanTri {
  float pv, pw;            // vs = pv e2x + bv e2y, ws = pw e2x + bw e2y (sign-adjusted)
  float ibv, ibw, ibu;     // 1 / bv, 1 / bw, 1 / (bv + bw)
  float lv, lw, uu;        // widened bounds: vs >= lv, ws >= lw, vs + ws <= uu
  float mv, mw, mu;        // widening of each bound's e2y crossing for its float evaluation
  float ax, clo, chi;      // vertex a's x; row y's e2y lies in [y + chi, y + clo] (widened for the row conversion)
  bool ok;                 // false: some slope is (nearly) 0, walk the whole box
};

// Triangle part.  e0*, e1*, d00, d01, d11 are the float values of the
// barycentric setup; rlo, ruhi the pre-reject bounds; x0..x1 the box columns,
// y0 the first row, ylen the box height.
//
// Error budget, in the units of the numerators.  Let S be the sum
// |d11| (mx |e0x| + my |e0y|) + |d01| (mx |e1x| + my |e1y|) for vs (mx, my:
// the largest |e2x|, |e2y| over the box; the matching sum for ws).  The
// pre-reject's float evaluation is within 2^-21 S of the linear form, and
// forming the coefficients pv, bv in float moves the linear form by at most
// 2^-22 S each over the box; the bounds are widened by 2^-18 S.  The
// crossing t = (l - a) / b is then computed with a float product and
// reciprocal: its error is below 2^-22 (|l| + 2 |a|) / |b| + 2^-24 |t|, and
// it is widened by four times that, taken at the largest |a| and |t| of the
// box (a crossing far outside the box stays outside).
TOMO_HD SpanTri span_setup(float ax, float ay, float e0x, float e0y, float e1x, float e1y, float d00, float d01,
                           float d11, bool dpos, float rlo, float ruhi, int x0, int x1, int y0, int ylen, float half)
{
  SpanTri T;
  const float pv = (d11 * e0x) - (d01 * e1x), bv = (d11 * e0y) - (d01 * e1y);
  const float pw = (d00 * e1x) - (d01 * e0x), bw = (d00 * e1y) - (d01 * e0y);
  T.pv = dpos ? pv : -pv;
  T.pw = dpos ? pw : -pw;
  const float sbv = dpos ? bv : -bv, sbw = dpos ? bw : -bw, sbu = sbv + sbw;
  T.ok = fabsf(sbv) > 1e-20f && fabsf(sbw) > 1e-20f && fabsf(sbu) > 1e-20f;
  T.ibv = recip_rn(T.ok ? sbv : 1.0f);
  T.ibw = recip_rn(T.ok ? sbw : 1.0f);
  T.ibu = recip_rn(T.ok ? sbu : 1.0f);
  const float ah = fabsf(half);
  const float mx = (float)(x1 - x0) + 2.0f + ah, my = (float)ylen + 2.0f + ah;
  const float a0x = fabsf(e0x), a0y = fabsf(e0y), a1x = fabsf(e1x), a1y = fabsf(e1y);
  const float k = 1.0f / 262144.0f;   // 2^-18 (twice the headroom the float forming of the bound needs)
  const float ev = k * (fabsf(d11) * (mx * a0x + my * a0y) + fabsf(d01) * (mx * a1x + my * a1y));
  const float ew = k * (fabsf(d00) * (mx * a1x + my * a1y) + fabsf(d01) * (mx * a0x + my * a0y));
  T.lv = sub_down(rlo, ev);
  T.lw = sub_down(rlo, ew);
  // vs + ws is rounded once more in float (|vs|, |ws| below |ruhi - rlo| there)
  T.uu = add_up(ruhi, (ev + ew) + k * (2.0f * fabsf(ruhi) + ev + ew));
  // crossing errors at the box's largest |a| and |t|
  const float amv = fabsf(T.pv) * mx, amw = fabsf(T.pw) * mx, tm = 2.0f * my;
  const float r20 = 1.0f / 1048576.0f;   // 2^-20
  T.mv = r20 * ((fabsf(T.lv) + 2.0f * amv) * fabsf(T.ibv) + tm);
  T.mw = r20 * ((fabsf(T.lw) + 2.0f * amw) * fabsf(T.ibw) + tm);
  T.mu = r20 * ((fabsf(T.uu) + 3.0f * (amv + amw)) * fabsf(T.ibu) + tm);
  T.ax = ax;
  // e2y = ((y + 0.001f) + half) - ay rounds three times, each within 2^-24
  // of a value below |y| + |half| + |ay| + 1 (y within the box), so it lies
  // within ey of y + c (c's own roundings and the float row conversion below
  // are inside ey too)
  const float ey = (fabsf((float)y0) + (float)ylen + ah + fabsf(ay) + tm + 2.0f) * (1.0f / 524288.0f);   // 2^-19
  const float c = (0.001f + half) - ay;
  T.clo = c + ey;
  T.chi = c - ey;
  return T;
}

// Rows [lo, hi] (lo > hi: none) of one column, within the box rows
// [y0, y0 + ylen - 1], whose centres the float pre-reject can pass.  px is
// the column's float pixel centre, the value the walk uses.
TOMO_HD void span_rows(const SpanTri& T, float px, int y0, int ylen, int& lo, int& hi)
{
  const float e2x = px - T.ax;   // the walk's float e2x
  const float av = T.pv * e2x, aw = T.pw * e2x, au = av + aw;
  const float tv = (T.lv - av) * T.ibv;   // vs >= lv: t >= tv for bv > 0, t <= tv for bv < 0
  const float tw = (T.lw - aw) * T.ibw;
  const float tu = (T.uu - au) * T.ibu;   // vs + ws <= uu: t <= tu for bu > 0, t >= tu for bu < 0
  float tlo = -3.0e38f, thi = 3.0e38f;
  if (T.ibv > 0.0f) tlo = fmaxf(tlo, tv - T.mv); else thi = fminf(thi, tv + T.mv);
  if (T.ibw > 0.0f) tlo = fmaxf(tlo, tw - T.mw); else thi = fminf(thi, tw + T.mw);
  if (T.ibu > 0.0f) thi = fminf(thi, tu + T.mu); else tlo = fmaxf(tlo, tu - T.mu);
  const float b0 = (float)y0, b1 = (float)(y0 + ylen - 1);
  const float l = fmaxf(ceilf(tlo - T.clo), b0), h = fminf(floorf(thi - T.chi), b1);
  if (!(l <= h)) { lo = 1; hi = 0; return; }
  lo = (int)l;
  hi = (int)h;
}

}  // namespace tomo
