// Shared device/host definitions of the B200 orientation-search engine.
//
// Arithmetic on this path reproduces the reference INT3 engine
// (cfms_tomo/Tomo_Shell_vc_src/cpu_src/STomoSh_INT3.cpp and Tomo_types.cpp)
// bit for bit: single-precision IEEE operations with one rounding each,
// written with __fadd_rn/__fmul_rn/__fdiv_rn so no FMA contraction can
// occur, and double precision exactly where the reference widens.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

namespace tomo {

// Slot capacity: the reference keeps at most 63 pixels per column
// (STomoVoxelSpaceInfo.cpp:47-51,214-218).
constexpr int kSlotCap = 63;

// Pixel type bits (Tomo_types.h:72-82).
enum : int {
  kAl = 1, kBe = 2, kSSB = 4, kSSA = 8, kSS = 16, kBed = 32,
  kVo = 64, kVss = 128, kTC = 256, kNVB = 512, kNVA = 1024
};

enum : int { kBedNone = 0, kBedBrim = 1, kBedRaft = 2, kBedSkirt = 3 };

// Fold records hold a column's (vo, vss) as two int16 and tc as one.  A
// column whose values leave [-32767, 32767] (or the narrower range a test
// asks for) writes the record kFoldEscaped
// (both halves -32768, which no packed pair produces) and appends its exact
// values, keyed by (orientation, record index), to the batch's escape table.
struct FoldEscape { int o, pos, vo, vss, tc, pad0, pad1, pad2; };
constexpr unsigned kFoldEscaped = 0x80008000u;
constexpr int kFoldEscapes = 1024;

// Per-orientation status bits.  The first three ask for the exact
// safe-mode re-run of that orientation; the rest are hard errors.
enum : int {
  kFlagStray = 1,      // a hit or fallback pixel landed outside its strip
  kFlagOverflow = 2,   // strip entry list exceeded shared memory
  kFlagBinCap = 4,     // triangle bin list exceeded its capacity
  kFlagGrid = 8,       // a slot index fell outside the grid (grid too small)
  kFlagSafeOverflow = 16,
  kFlagCap = 32,       // a column exceeded the 63-pixel cap: needs first-come priorities
  kFlagFoldRange = 64, // column values past 16 bits overflowed the batch's escape table
};
// Results of an orientation flagged with any of these are not written.
constexpr int kFlagRedo = kFlagStray | kFlagOverflow | kFlagBinCap | kFlagCap;

// Bed bookkeeping per slot (GenerateBed / IsBedCandidate, STomoSh_INT3.cpp:1331-1443).
enum : uint8_t {
  kBfOcc = 1,     // slot holds at least one pixel after voxelization
  kBfTouch = 2,   // last pixel at z == 0 with alpha/beta/SSA/SS type: floor contact
  kBfPoss = 4,    // a bed pixel may go here
  kBfLand = 8,    // a bed pixel would be stored (room left or key (1,0) present)
  kBfSelfR = 16,  // raft pixel appended here hides this slot's floor contact afterwards
};

// Accumulator lanes per orientation (int64).
enum : int {
  kAccVo = 0, kAccVss, kAccVtc, kAccAbsVss, kAccAbsVtc, kAccEntries, kAccColumns, kAccFoldN, kAccLanes
};

struct EngineParams {
  // mesh (raw, as given by the caller)
  const float4* vpos;   // [nV] x, y, z, 0
  const float4* vnrm;   // [nV] nx, ny, nz, 0
  const int4* tri;      // [nT] a, b, c, 0
  int nV, nT;

  // orientations
  const float* rot;     // [nYPR][9] rotation matrices (host-computed)
  const int* ori;       // [Bo] orientation id per batch slot
  int Bo;

  float cx, cy, cz;     // AABB centre of the raw vertices
  float bed_outer, bed_inner;
  int bed_type, bed_r;
  float bed_thickness;

  // grid
  int G;                // square grid edge; slot id = x * G + y
  int H;                // strip height in x columns
  int S;                // number of strips = ceil(G / H)
  int mode;             // 0 normal, 1 safe, 2 normal with priorities
  int variant;          // strip configuration (launch accounting only)

  // raster constants
  float half;           // dVoxel * 0.5f
  float shell_off;      // float(int(shell_thickness + 0.999f))
  int twin;             // bShellMesh && shell_thickness > 0.001f
  float vmax;           // largest float <= 1.0 + double(0.001f)
  float thr;            // float(-sin(theta_c))
  int explicit_ss;

  // shared-memory layout of the strip kernel
  int ent_cap;          // entries per strip CTA

  // work buffers
  float4* xf;           // [Bo][nV] rotated x, y, z, n.z
  unsigned* minkey;     // [Bo][4] order-preserving keys of AABB minima
  unsigned* trange;     // [Bo][nT] packed strip range of each triangle (k_bin_count -> k_bin_fill)
  int* bin_off;         // [Bo][S + 1]
  int* bin_cur;         // [Bo][S]
  int* bins;            // [Bo][bin_cap]
  int bin_cap;

  // per-batch results
  long long* acc;       // [Bo][kAccLanes]
  int* flags;           // [Bo]
  int* bbox;            // [Bo][4] min x, min y, max x, max y of occupied slots
  uint8_t* bedf;        // [Bo][G*G]
  int* foldcnt;         // [Bo][S]
  unsigned* foldp;      // [Bo][G*G] (vo, vss) of each occupied column as two int16, in slot order per strip
  short* foldtc;        // [Bo][G*G] tc of each occupied column (implicit support only, else null)
  FoldEscape* foldx;    // [kFoldEscapes] columns whose values do not fit 16 bits (record kFoldEscaped)
  int* foldxn;          // entries appended to foldx in this batch
  int fold_lim;         // largest |value| a packed record holds (32767; lower only to test the escape table)
  int* foldmeta;        // [Bo][S][8] per strip: sum vo, vss, tc, |vss|, |tc|

  // per-orientation outputs (indexed by orientation id)
  long long* out_vo;
  long long* out_vss;
  long long* out_vtc;
  float* out_vof;
  float* out_vssf;
  float* out_vtcf;
  int* out_nbed;
  int* out_flags;
  long long* out_entries;
  long long* out_columns;

  // optional dense per-column dump for one batch slot (debug / parity)
  int dump_slot;        // batch slot to dump, or -1
  int* dump_cols;       // [G*G][8]: n_distinct, n_final, vo, vss, tc, last_z, last_type, flags
  unsigned* dump_keys;  // [G*G][64] kept (z, nz) keys in column order, or null
  short* dump_types;    // [G*G][64] their final types
};

// Kernel kinds for launch accounting.
enum : int { kKReset = 0, kKRotate, kKCount, kKScan, kKFill, kKStrip, kKBed, kKFold, kKStripRedo, kKinds };

// Host-side launch log: launch counts per kernel kind and, when timing is
// on, one event pair per launch recorded on the launching stream.
struct LaunchLog {
  struct Span { int kind; cudaEvent_t start, stop; };
  bool timing = false;
  long long launches[kKinds] = {0};
  double ms[kKinds] = {0};
  long long timed[kKinds] = {0};
  std::vector<Span> pending;
  std::vector<cudaEvent_t> pool;
  size_t next = 0;

  cudaEvent_t take_event()
  {
    if (next == pool.size()) {
      cudaEvent_t e = nullptr;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[next++];
  }
  // Fold the pending spans into ms[] (the streams must be idle).
  void collect()
  {
    for (const Span& s : pending) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, s.start, s.stop) == cudaSuccess) { ms[s.kind] += t; timed[s.kind]++; }
    }
    pending.clear();
    next = 0;
  }
  void reset()
  {
    pending.clear();
    next = 0;
    for (int k = 0; k < kKinds; k++) { launches[k] = 0; ms[k] = 0; timed[k] = 0; }
  }
  void destroy()
  {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
    pool.clear();
    pending.clear();
    next = 0;
  }
};

}  // namespace tomo
