// Host side of the B200 orientation-search engine and its C-ABI.
//
// The C-ABI mirrors the reference DLL exports (Tomo_Shell_vc_src/Tomo_Shell2026.h:19-35):
// TomoSh_CUDA takes the same ten pointers and returns optID; the getters return
// library-owned buffers valid until the next call or OnDestroy.  Errors are
// returned as negative codes (tomoGetLastError / tomoGetLastErrorString)
// instead of the reference's exit(0) on CUDA failure (cuda_src/CUDA_types.cuh:112-118).
//
// Work split: rotation matrices, the shadow threshold and the mass model are
// evaluated on the host with the same C library calls as the reference
// (SMatrix4f::YPR, STomoSh_INT3.cpp:756, STomoVolMassInfo::VolToMass), so those
// floats are bit-identical by construction; everything per vertex, triangle,
// pixel and column runs in the kernels of tomo_kernels.cu.
#include "tomo_common.cuh"
#include "tomo_mlp.cuh"
#include "../../include/tomo_b200.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace tomo {

size_t strip_smem_bytes(int mode, int H, int G, int ent_cap);
size_t strip_four_per_sm_budget();
cudaError_t configure_kernels(size_t normal_smem, size_t safe_smem, size_t prio_smem);
cudaError_t launch_batch(const EngineParams& p, cudaStream_t main, size_t strip_smem, LaunchLog* L);
cudaError_t launch_fold(const EngineParams& p, cudaStream_t side, LaunchLog* L);
cudaError_t launch_bin_count(const EngineParams& p, cudaStream_t main, LaunchLog* L);
cudaError_t launch_after_count(const EngineParams& p, cudaStream_t main, size_t strip_smem, LaunchLog* L);
cudaError_t launch_fill(const EngineParams& p, cudaStream_t s, LaunchLog* L);
cudaError_t launch_strip_bed(const EngineParams& p, cudaStream_t main, size_t strip_smem, LaunchLog* L);
cudaError_t launch_dump_scan(const int* cols8, int GG, int* off, int* totals, cudaStream_t s);
cudaError_t launch_zero_ids(int* out, const int* ids, int n, cudaStream_t s);
cudaError_t launch_read_probe(const void* buf, long long bytes, int reps, int blocks, cudaStream_t s);
cudaError_t launch_gather_outputs(const long long* vo, const long long* vss, const long long* vtc, const long long* ent,
                                  const long long* col, const float* vof, const float* vssf, const float* vtcf,
                                  const int* nbed, const int* flags, const int* ids, int n, long long* stage,
                                  cudaStream_t s);
cudaError_t launch_scatter_rot(float* rot, const float* compact, const int* ids, int n, cudaStream_t s);
cudaError_t launch_dump_gather(const int* cols8, const unsigned* keys64, const short* types64, int GG, const int* off,
                               int* cols9, unsigned* keys, short* types, cudaStream_t s);

namespace {

std::mutex g_mutex;
int g_last_error = 0;
std::string g_last_error_str;

int set_error(int code, const std::string& msg)
{
  g_last_error = code;
  g_last_error_str = msg;
  return code;
}

#define TOMO_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return set_error(TOMO_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TOMO_TRY(call)        \
  do {                        \
    const int rc_ = (call);   \
    if (rc_ != 0) return rc_; \
  } while (0)

// ------------------------------------------------ host arithmetic (bit-exact with the reference)

// SMatrix4f::YPR (cpu_src/SMatrix4f.cpp:213-240), 3x3 block row-major.
void rotation(float ga, float be, float al, float R[9])
{
  const float cos_al = cosf(al), cos_be = cosf(be), cos_ga = cosf(ga);
  const float sin_al = sinf(al), sin_be = sinf(be), sin_ga = sinf(ga);
  R[0] = cos_al * cos_be;
  R[1] = cos_al * sin_be * sin_ga - sin_al * cos_ga;
  R[2] = cos_al * sin_be * cos_ga + sin_al * sin_ga;
  R[3] = sin_al * cos_be;
  R[4] = sin_al * sin_be * sin_ga + cos_al * cos_ga;
  R[5] = sin_al * sin_be * cos_ga - cos_al * sin_ga;
  R[6] = -sin_be;
  R[7] = cos_be * sin_ga;
  R[8] = cos_be * cos_ga;
}

struct Params {
  float dVoxel, theta_c, surface_area, wall, Fcore, Fclad, Fss, Css, rho;
  float bed_inner, bed_outer, bed_thickness;
  int explicit_ss, shell, n_tri, n_vtx, n_ypr, bed_type;
  float shell_thickness;
};

// S3DPrinterInfo::Set (cpu_src/S3DPrinterInfo.cpp:130-144)
Params read_params(const float* f, const int* i)
{
  Params p;
  p.dVoxel = f[0]; p.theta_c = f[1]; p.surface_area = f[2]; p.wall = f[3];
  p.Fcore = f[4]; p.Fclad = f[5]; p.Fss = f[6]; p.Css = f[7]; p.rho = f[8];
  p.bed_inner = f[9]; p.bed_outer = f[10]; p.bed_thickness = f[11];
  p.explicit_ss = ((float)i[1] > 0.001f);
  p.shell = ((float)i[2] > 0.001f);
  p.shell_thickness = (float)i[10] * 0.001f;
  p.n_tri = i[4]; p.n_vtx = i[5]; p.n_ypr = i[6]; p.bed_type = i[9];
  return p;
}

// STomoVolMassInfo::VolToMass (cpu_src/STomoVolMassInfo.cpp:42-80); vm in
// the 22-float vm_info layout (STomoVolMassInfo.h:19-33).
void vol_to_mass(const Params& P, float* vm)
{
  const float Vss = vm[4], Vo = vm[8], Vbed = vm[11];
  const float Vo_clad = P.surface_area * P.wall;
  const float Vo_core = Vo - Vo_clad;
  const float Mo_clad = Vo_clad * P.Fclad * P.rho;
  const float Mo_core = Vo_core * P.Fcore * P.rho;
  const float Mo = Mo_core + Mo_clad;
  float Vss_clad = 0.f, Vss_core = 0.f, Ass_clad = 0.f, Mss_clad = 0.f, Mss_core = 0.f, Mss = 0.f;
  if (P.explicit_ss) {
    if (Vss > 0.001f) {
      const float radius = powf(Vss / (4.f / 3.f * 3.141592f), 1.f / 3.f);
      Ass_clad = (float)(4. * 3.141592 * (double)radius * (double)radius);
      Vss_clad = Ass_clad * P.wall;
      if (Vss_clad > Vss) Vss_clad = Vss;
      Vss_core = Vss - Vss_clad;
      Mss_clad = Vss_clad * P.Fclad * P.rho;
      Mss_core = Vss_core * P.Fcore * P.rho;
      Mss = Mss_core + Mss_clad;
    }
  } else {
    Mss = Vss * P.Fss * P.Css * P.rho;
  }
  const float Mbed = Vbed * P.wall * P.rho;
  Mss += Mbed;
  vm[5] = Vss_clad; vm[6] = Vss_core; vm[7] = Ass_clad;
  vm[9] = Vo_clad; vm[10] = Vo_core;
  vm[12] = Mbed;
  vm[13] = Mss; vm[14] = Mss_clad; vm[15] = Mss_core;
  vm[16] = Mo; vm[17] = Mo_clad; vm[18] = Mo_core;
  vm[19] = Mo + Mss;
}

// _find1stOptimal (Tomo_Shell2026.cpp:89-97)
int first_optimal(int n, const float* mss)
{
  if (n <= 1) return 0;
  int idx = 0;
  float best = 1e5f;
  for (int i = 0; i < n; i++)
    if (mss[i] < best) { best = mss[i]; idx = i; }
  return idx;
}

float largest_float_not_above(double c)
{
  float f = (float)c;
  while ((double)f > c) f = nextafterf(f, -INFINITY);
  while ((double)nextafterf(f, INFINITY) <= c) f = nextafterf(f, INFINITY);
  return f;
}

template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  cudaError_t reserve(size_t count)
  {
    if (count <= n && ptr) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr; n = 0;
    cudaError_t e = cudaMalloc((void**)&ptr, sizeof(T) * (count ? count : 1));
    if (e == cudaSuccess) n = count;
    return e;
  }
  void release() { if (ptr) cudaFree(ptr); ptr = nullptr; n = 0; }
};

// Largest slot grid edge (columns of the rotated footprint at the voxel pitch).
constexpr int kMaxGrid = 4096;

// Orientations the last tomoSweepStatic call re-ran, per strip configuration.
int g_static_reruns[5];

// Proposal source of tomoSurrogateSearch: 0 the trained network, 1 bilinear
// interpolation of the exact coarse values (the search without the network),
// 2 the mean of the two.
int g_proposal = 0;

struct BatchSet {   // per-batch buffers read by the fold, double-buffered
  DevBuf<long long> acc;
  DevBuf<int> flags;
  DevBuf<int> foldcnt;
  DevBuf<unsigned> foldp;
  DevBuf<short> foldtc;
  DevBuf<FoldEscape> foldx;
  DevBuf<int> foldxn;
  DevBuf<int> foldmeta;
  cudaEvent_t folded = nullptr;
};

struct PrepSet {    // a batch's rotated vertices and strip bins (binning -> strips)
  DevBuf<float4> xf;
  DevBuf<unsigned> minkey;
  DevBuf<unsigned> trange;
  DevBuf<int> bin_off, bin_cur, bins, bbox;
  DevBuf<uint8_t> bedf;
  cudaEvent_t ready = nullptr;
  void release()
  {
    xf.release(); minkey.release(); trange.release(); bin_off.release(); bin_cur.release(); bins.release();
    bbox.release(); bedf.release();
  }
};

}  // namespace

// ------------------------------------------------ engine

// Streams and batch work buffers, shared by every mesh of a multi-mesh sweep
// (one Workspace per Engine for the single-mesh C-ABI).  Buffers only grow.
struct Workspace {
  int device = -1;
  cudaStream_t main = nullptr, side = nullptr, binning = nullptr;
  cudaEvent_t ev_ready = nullptr;
  size_t smem_optin = 0;
  PrepSet prep[2];   // prep[0] is also the single set of the one-batch paths
  BatchSet set[2];
  DevBuf<int> dump_cols;
  DevBuf<unsigned> dump_keys;
  DevBuf<short> dump_types;
  DevBuf<int> dump_off, dump_tot, dump_ccols;
  DevBuf<unsigned> dump_ckeys;
  DevBuf<short> dump_ctypes;
  LaunchLog log;

  int init()
  {
    if (main) return 0;
    int dev = 0;
    TOMO_CUDA(cudaGetDevice(&dev));
    device = dev;
    TOMO_CUDA(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
    TOMO_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    TOMO_CUDA(cudaStreamCreateWithFlags(&binning, cudaStreamNonBlocking));
    TOMO_CUDA(cudaEventCreateWithFlags(&ev_ready, cudaEventDisableTiming));
    for (auto& s : set) TOMO_CUDA(cudaEventCreateWithFlags(&s.folded, cudaEventDisableTiming));
    for (auto& q : prep) TOMO_CUDA(cudaEventCreateWithFlags(&q.ready, cudaEventDisableTiming));
    int optin = 0;
    TOMO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    smem_optin = (size_t)optin;
    return 0;
  }

  void release()
  {
    for (auto& q : prep) q.release();
    for (auto& s : set) { s.acc.release(); s.flags.release(); s.foldcnt.release(); s.foldp.release(); s.foldtc.release(); s.foldx.release(); s.foldxn.release(); s.foldmeta.release(); }
    dump_cols.release(); dump_keys.release(); dump_types.release();
    dump_off.release(); dump_tot.release(); dump_ccols.release(); dump_ckeys.release(); dump_ctypes.release();
    log.destroy();
    if (main) { cudaStreamDestroy(main); main = nullptr; }
    if (side) { cudaStreamDestroy(side); side = nullptr; }
    if (binning) { cudaStreamDestroy(binning); binning = nullptr; }
    for (auto& q : prep) if (q.ready) { cudaEventDestroy(q.ready); q.ready = nullptr; }
    if (ev_ready) { cudaEventDestroy(ev_ready); ev_ready = nullptr; }
    for (auto& s : set) if (s.folded) { cudaEventDestroy(s.folded); s.folded = nullptr; }
  }
};

// One mesh: its device arrays, orientations, outputs and host results; the
// streams and work buffers are the Workspace's (bound by reference).
struct Engine {
  Workspace& W;
  bool owns_ws;
  int& device;
  cudaStream_t& main;
  cudaStream_t& side;
  cudaEvent_t& ev_ready;
  size_t& smem_optin;
  DevBuf<float4>& xf;
  DevBuf<unsigned>& minkey;
  DevBuf<unsigned>& trange;
  DevBuf<int>& bin_off;
  DevBuf<int>& bin_cur;
  DevBuf<int>& bins;
  DevBuf<int>& bbox;
  DevBuf<uint8_t>& bedf;
  BatchSet (&set)[2];
  DevBuf<int>& dump_cols;
  DevBuf<unsigned>& dump_keys;
  DevBuf<short>& dump_types;
  DevBuf<int>& dump_off;
  DevBuf<int>& dump_tot;
  DevBuf<int>& dump_ccols;
  DevBuf<unsigned>& dump_ckeys;
  DevBuf<short>& dump_ctypes;
  LaunchLog& log;

  explicit Engine(Workspace& w, bool owns = false)
      : W(w), owns_ws(owns), device(w.device), main(w.main), side(w.side), ev_ready(w.ev_ready),
        smem_optin(w.smem_optin), xf(w.prep[0].xf), minkey(w.prep[0].minkey), trange(w.prep[0].trange),
        bin_off(w.prep[0].bin_off), bin_cur(w.prep[0].bin_cur), bins(w.prep[0].bins), bbox(w.prep[0].bbox),
        bedf(w.prep[0].bedf), set(w.set), dump_cols(w.dump_cols),
        dump_keys(w.dump_keys), dump_types(w.dump_types), dump_off(w.dump_off), dump_tot(w.dump_tot),
        dump_ccols(w.dump_ccols), dump_ckeys(w.dump_ckeys), dump_ctypes(w.dump_ctypes), log(w.log)
  {
  }
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // mesh and orientations
  DevBuf<float4> vpos, vnrm;
  DevBuf<int4> tri;
  DevBuf<float> rot;
  DevBuf<int> ori;
  // outputs
  DevBuf<long long> o_vo, o_vss, o_vtc, o_ent, o_col;
  DevBuf<float> o_vof, o_vssf, o_vtcf;
  DevBuf<int> o_nbed, o_flags;
  // learned-proposal search: orientations, network features and
  // predictions of the grid, kept between searches (they only grow)
  DevBuf<float> srch_ypr, srch_x, srch_y;
  // subset fetch (see fetch_subset) and lazy rotations (see ensure_rot)
  DevBuf<int> sub_ids;
  DevBuf<long long> sub_stage;
  std::vector<int> sub_host;
  int sub_n = 0;
  std::vector<float> h_ypr;
  std::vector<char> rot_ready;

  // host results of the last sweep
  Params P{};
  int nYPR = 0, G = 0, H = 0, S = 0, ent_cap = 0;
  int batch = 256;
  int force_h = 0;        // test hook: strip height override
  int force_safe = 0;     // test hook: run every orientation in safe mode
  int normal_smem = 0;    // shared-memory budget of a normal strip CTA (0 = four CTAs per SM)
  int export_pixels = 1;  // rebuild the best orientation's pixels and vm_info (TomoSh_CUDA tail)
  int adaptive = 1;       // raise the entry budget after overflowing early batches (full sweeps)
  int fold_lim = 32767;   // largest |column value| of a packed fold record (TOMO_OPT_FOLD_LIMIT)
  int adapt_smem = 0, adapt_h = 0;   // configuration adapted to by an earlier sweep of this upload
  int adapt_cfg = 0;                  // 4 once a sweep of this upload switched to priority strips
  int start_cfg = 0;                  // 4: every sweep starts in priority strips (set by the batch autotuner)
  float cx = 0, cy = 0, cz = 0;
  std::vector<float> h_rot;
  std::vector<float> h_vtx;   // the caller's vertices, kept for mat4x4 of a later export
  std::vector<long long> vo64, vss64, vtc64, entries, columns;
  std::vector<float> vof, vssf, vtcf, Mo, Mss, Vtc;
  std::vector<int> nbed, flags;
  float volmass[22] = {0};
  float mat4x4[16] = {0};
  double last_kernel_ms = 0.0;
  int n_safe = 0;
  int n_redo[5] = {0, 0, 0, 0, 0};
  int H_sweep = 0;        // strip height of the last normal sweep

  int init() { return W.init(); }

  // Frees this mesh's buffers, and the workspace when the engine owns it.
  void release()
  {
    vpos.release(); vnrm.release(); tri.release(); rot.release(); ori.release();
    sub_ids.release(); sub_stage.release();
    srch_ypr.release(); srch_x.release(); srch_y.release();
    o_vo.release(); o_vss.release(); o_vtc.release(); o_ent.release(); o_col.release();
    o_vof.release(); o_vssf.release(); o_vtcf.release(); o_nbed.release(); o_flags.release();
    if (owns_ws) W.release();
  }

  // Grid edge: the reference grid is 256 x 256 (STomoVoxelSpaceInfo.h:10).
  // Keep it whenever the rotated mesh fits, so every bounded result
  // (including the bed window clipping at the grid edge) is the reference's;
  // grow it otherwise (the reference would write out of bounds there).
  int choose_grid(const float* vtx, int nV)
  {
    double r2 = 0.0;
    for (int v = 0; v < nV; v++) {
      const double dx = (double)vtx[v * 3 + 0] - cx, dy = (double)vtx[v * 3 + 1] - cy, dz = (double)vtx[v * 3 + 2] - cz;
      r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
    }
    const double span = 2.0 * std::sqrt(r2) * 1.004 + std::max(0.0, (double)P.bed_outer) + 6.0;
    if (span <= 256.0) return 256;
    return (int)span + (int)std::max(0.0f, P.bed_outer) + 2;
  }

  // Strip configurations.
  //   0 normal     : H0-column strips, ~55 KB of shared memory (four CTAs
  //                  per SM), entries without priorities; H0 is the tallest
  //                  strip with room for two entries per slot;
  //   1 safe       : H0-column strips, whole-box evaluation, priorities,
  //                  all opt-in shared memory;
  //   2 big normal : configuration 0 semantics with all opt-in shared memory
  //                  (orientations whose strip lists overflowed);
  //   3 narrow safe: safe mode with one-column strips (last resort);
  //   4 priorities : configuration 0 strips whose entries also carry their
  //                  first-come priority, all opt-in shared memory, for
  //                  orientations where a column passed the 63-pixel cap.
  struct StripCfg { int H, S, C; size_t smem; int mode; };
  StripCfg cfg[5];

  void plan_strips()
  {
    const size_t optin = smem_optin ? smem_optin : 232448;
    // default: the largest budget that keeps four CTAs on an SM (~55 KB on B200)
    const size_t four = strip_four_per_sm_budget();
    const size_t budget0 = std::min<size_t>(optin - 2048, normal_smem ? (size_t)normal_smem : (four ? four : 73728));
    // the strip kernel also holds ~0.7 KB of static shared memory
    const size_t budget1 = std::min<size_t>(optin, 227 * 1024) - 2048;
    int h0 = 1;
    for (int h : {8, 4, 2, 1}) {
      if (force_h && h != force_h) continue;
      const size_t fixed = strip_smem_bytes(0, h, G, 0);
      if (fixed + 6 * 256 >= budget0) continue;
      const int cap = (int)std::min<size_t>((budget0 - fixed) / 6 - 16, 32767);
      if (force_h || cap >= 2 * h * G) { h0 = h; break; }
    }
    auto make = [&](int mode, int h, size_t budget) {
      StripCfg c;
      c.mode = mode; c.H = h; c.S = (G + h - 1) / h;
      const size_t per = mode == 0 ? 6 : 15;
      const size_t fixed = strip_smem_bytes(mode, h, G, 0);
      c.C = (int)std::min<size_t>(budget > fixed + 32 * per ? (budget - fixed) / per - 16 : 16, 32767);
      c.smem = strip_smem_bytes(mode, h, G, c.C);
      return c;
    };
    cfg[0] = make(0, h0, budget0);
    cfg[1] = make(1, h0, budget1);
    cfg[2] = make(0, h0, budget1);
    cfg[3] = make(1, 1, budget1);
    cfg[4] = make(2, h0, budget1);
  }

  void choose_strips(int c)
  {
    H = cfg[c].H; S = cfg[c].S; ent_cap = cfg[c].C;
  }

  int configure()
  {
    TOMO_CUDA(configure_kernels(std::max(cfg[0].smem, cfg[2].smem), std::max(cfg[1].smem, cfg[3].smem), cfg[4].smem));
    return 0;
  }

  int upload(const float* f32, const int* i32, const float* ypr, const int* tri_h, const float* vtx,
             const float* vnrm_h, bool lazy_rot = false)
  {
    P = read_params(f32, i32);
    if (P.n_tri < 0 || P.n_vtx < 0 || P.n_ypr < 0) return set_error(TOMO_ERR_ARG, "negative size in Int32Info");
    if (P.n_ypr > 0 && ypr == nullptr) return set_error(TOMO_ERR_ARG, "YPR is null");
    if (P.n_tri > 0 && (tri_h == nullptr || vtx == nullptr || vnrm_h == nullptr))
      return set_error(TOMO_ERR_ARG, "mesh array is null");
    for (int t = 0; t < P.n_tri * 3; t++)
      if (tri_h[t] < 0 || tri_h[t] >= P.n_vtx) return set_error(TOMO_ERR_ARG, "triangle index out of range");
    for (int k = 0; k < P.n_vtx * 3; k++)
      if (!std::isfinite(vtx[k]) || !std::isfinite(vnrm_h[k])) return set_error(TOMO_ERR_ARG, "non-finite vertex or normal");
    for (int k = 0; k < P.n_ypr * 3; k++)
      if (!std::isfinite(ypr[k])) return set_error(TOMO_ERR_ARG, "non-finite orientation");
    if (!std::isfinite(P.dVoxel) || !std::isfinite(P.bed_outer) || !std::isfinite(P.theta_c) || P.bed_outer < 0.f ||
        P.bed_outer > 1000.f)
      return set_error(TOMO_ERR_ARG, "bad printer parameters");
    nYPR = P.n_ypr;
    adapt_smem = adapt_h = adapt_cfg = 0;
    // AABB centre of the raw vertices (STomoAABB3Df.cpp:58-72)
    float mn[3] = {1e5f, 1e5f, 1e5f}, mx[3] = {-1e5f, -1e5f, -1e5f};
    for (int v = 0; v < P.n_vtx; v++)
      for (int k = 0; k < 3; k++) {
        const float d = vtx[v * 3 + k];
        mn[k] = (mn[k] <= d) ? mn[k] : d;
        mx[k] = (mx[k] >= d) ? mx[k] : d;
      }
    cx = (float)((double)(mn[0] + mx[0]) * 0.5);
    cy = (float)((double)(mn[1] + mx[1]) * 0.5);
    cz = (float)((double)(mn[2] + mx[2]) * 0.5);
    G = choose_grid(vtx, P.n_vtx);
    if (G > kMaxGrid) return set_error(TOMO_ERR_CAPACITY, "mesh extent exceeds the supported slot grid");
    plan_strips();

    std::vector<float4> hp(std::max(P.n_vtx, 1)), hn(std::max(P.n_vtx, 1));
    for (int v = 0; v < P.n_vtx; v++) {
      hp[v] = make_float4(vtx[v * 3 + 0], vtx[v * 3 + 1], vtx[v * 3 + 2], 0.f);
      hn[v] = make_float4(vnrm_h[v * 3 + 0], vnrm_h[v * 3 + 1], vnrm_h[v * 3 + 2], 0.f);
    }
    std::vector<int4> ht(std::max(P.n_tri, 1));
    for (int t = 0; t < P.n_tri; t++) ht[t] = make_int4(tri_h[t * 3 + 0], tri_h[t * 3 + 1], tri_h[t * 3 + 2], 0);
    h_vtx.assign(vtx, vtx + (size_t)P.n_vtx * 3);
    h_rot.assign((size_t)std::max(nYPR, 1) * 9, 0.f);
    rot_ready.assign((size_t)std::max(nYPR, 1), lazy_rot ? 0 : 1);
    if (lazy_rot) h_ypr.assign(ypr, ypr + (size_t)nYPR * 3);
    else
      for (int i = 0; i < nYPR; i++) rotation(ypr[i * 3 + 0], ypr[i * 3 + 1], ypr[i * 3 + 2], &h_rot[(size_t)i * 9]);
    std::vector<int> hori(std::max(nYPR, 1));
    for (int i = 0; i < nYPR; i++) hori[i] = i;

    TOMO_CUDA(vpos.reserve(hp.size())); TOMO_CUDA(vnrm.reserve(hn.size()));
    TOMO_CUDA(tri.reserve(ht.size())); TOMO_CUDA(rot.reserve(h_rot.size())); TOMO_CUDA(ori.reserve(hori.size()));
    TOMO_CUDA(cudaMemcpyAsync(vpos.ptr, hp.data(), sizeof(float4) * hp.size(), cudaMemcpyHostToDevice, main));
    TOMO_CUDA(cudaMemcpyAsync(vnrm.ptr, hn.data(), sizeof(float4) * hn.size(), cudaMemcpyHostToDevice, main));
    TOMO_CUDA(cudaMemcpyAsync(tri.ptr, ht.data(), sizeof(int4) * ht.size(), cudaMemcpyHostToDevice, main));
    if (!lazy_rot)
      TOMO_CUDA(cudaMemcpyAsync(rot.ptr, h_rot.data(), sizeof(float) * h_rot.size(), cudaMemcpyHostToDevice, main));
    TOMO_CUDA(cudaMemcpyAsync(ori.ptr, hori.data(), sizeof(int) * hori.size(), cudaMemcpyHostToDevice, main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    return 0;
  }

  EngineParams base_params(int mode)
  {
    EngineParams p;
    std::memset(&p, 0, sizeof(p));
    p.vpos = vpos.ptr; p.vnrm = vnrm.ptr; p.tri = tri.ptr; p.nV = P.n_vtx; p.nT = P.n_tri;
    p.rot = rot.ptr;
    p.cx = cx; p.cy = cy; p.cz = cz;
    p.bed_outer = P.bed_outer; p.bed_inner = P.bed_inner; p.bed_type = P.bed_type;
    p.bed_r = (int)P.bed_outer; p.bed_thickness = P.bed_thickness;
    p.G = G; p.H = H; p.S = S; p.mode = mode;
    p.half = P.dVoxel * 0.5f;
    p.shell_off = (float)(int)(P.shell_thickness + 0.999f);
    p.twin = (P.shell && P.shell_thickness > 0.001f) ? 1 : 0;
    p.vmax = largest_float_not_above(1.0 + (double)0.001f);
    p.thr = (float)(-1.0 * (double)sinf(P.theta_c));   // STomoSh_INT3.cpp:756
    p.explicit_ss = P.explicit_ss;
    p.ent_cap = ent_cap;
    p.out_vo = o_vo.ptr; p.out_vss = o_vss.ptr; p.out_vtc = o_vtc.ptr;
    p.out_vof = o_vof.ptr; p.out_vssf = o_vssf.ptr; p.out_vtcf = o_vtcf.ptr;
    p.out_nbed = o_nbed.ptr; p.out_flags = o_flags.ptr; p.out_entries = o_ent.ptr; p.out_columns = o_col.ptr;
    p.dump_slot = -1;
    p.fold_lim = fold_lim;
    return p;
  }

  int reserve_batch(int Bo, int bin_cap, int nprep = 1)
  {
    const size_t GG = (size_t)G * G;
    for (int q = 0; q < nprep; q++) {
      PrepSet& b = W.prep[q];
      TOMO_CUDA(b.xf.reserve((size_t)Bo * std::max(P.n_vtx, 1)));
      TOMO_CUDA(b.minkey.reserve((size_t)Bo * 4));
      TOMO_CUDA(b.trange.reserve((size_t)Bo * std::max(P.n_tri, 1)));
      TOMO_CUDA(b.bin_off.reserve((size_t)Bo * (S + 1)));
      TOMO_CUDA(b.bin_cur.reserve((size_t)Bo * S));
      TOMO_CUDA(b.bins.reserve((size_t)Bo * bin_cap));
      TOMO_CUDA(b.bbox.reserve((size_t)Bo * 4));
      TOMO_CUDA(b.bedf.reserve((size_t)Bo * GG));
    }
    for (auto& s : set) {
      TOMO_CUDA(s.acc.reserve((size_t)Bo * kAccLanes));
      TOMO_CUDA(s.flags.reserve((size_t)Bo));
      TOMO_CUDA(s.foldcnt.reserve((size_t)Bo * S));
      TOMO_CUDA(s.foldp.reserve((size_t)Bo * GG));
      if (!P.explicit_ss) TOMO_CUDA(s.foldtc.reserve((size_t)Bo * GG));
      TOMO_CUDA(s.foldx.reserve(kFoldEscapes));
      TOMO_CUDA(s.foldxn.reserve(1));
      TOMO_CUDA(s.foldmeta.reserve((size_t)Bo * S * 8));
    }
    return 0;
  }

  int reserve_outputs()
  {
    const size_t n = (size_t)std::max(nYPR, 1);
    TOMO_CUDA(o_vo.reserve(n)); TOMO_CUDA(o_vss.reserve(n)); TOMO_CUDA(o_vtc.reserve(n));
    TOMO_CUDA(o_ent.reserve(n)); TOMO_CUDA(o_col.reserve(n));
    TOMO_CUDA(o_vof.reserve(n)); TOMO_CUDA(o_vssf.reserve(n)); TOMO_CUDA(o_vtcf.reserve(n));
    TOMO_CUDA(o_nbed.reserve(n)); TOMO_CUDA(o_flags.reserve(n));
    return 0;
  }

  void bind_batch(EngineParams& p, int Bo, int bin_cap, int which, int first, int q = 0)
  {
    const PrepSet& b = W.prep[q];
    p.Bo = Bo;
    p.ori = ori.ptr + first;
    p.xf = b.xf.ptr; p.minkey = b.minkey.ptr; p.trange = b.trange.ptr;
    p.bin_off = b.bin_off.ptr; p.bin_cur = b.bin_cur.ptr; p.bins = b.bins.ptr; p.bin_cap = bin_cap;
    p.bbox = b.bbox.ptr; p.bedf = b.bedf.ptr;
    p.acc = set[which].acc.ptr; p.flags = set[which].flags.ptr;
    p.foldcnt = set[which].foldcnt.ptr; p.foldp = set[which].foldp.ptr; p.foldmeta = set[which].foldmeta.ptr;
    p.foldtc = p.explicit_ss ? nullptr : set[which].foldtc.ptr;
    p.foldx = set[which].foldx.ptr; p.foldxn = set[which].foldxn.ptr;
  }

  // All orientations in configuration 0, asynchronously on `main`.  With
  // `ids`, only the n_ids orientations listed in that device array.
  int sweep_device(const int* ids = nullptr, int n_ids = 0)
  {
    const int n = ids ? n_ids : nYPR;
    if (n == 0 || P.n_tri == 0) return 0;
    // a full sweep starts from the configuration an earlier sweep of this
    // upload adapted to (see adapt_after below)
    const int user_smem = normal_smem, user_h = force_h;
    const bool adapt = adaptive && !ids;
    if (adapt && adapt_smem) { normal_smem = adapt_smem; force_h = adapt_h; plan_strips(); }
    const int rc = sweep_batches(ids, n, adapt);
    if (adapt && (normal_smem != user_smem || force_h != user_h)) {
      normal_smem = user_smem; force_h = user_h; plan_strips();
    }
    return rc;
  }

  // After an early batch: if more than a fifth of its orientations overflowed
  // their strip lists, give the rest of the sweep the next larger entry
  // budget at the same strip height (one host wait per check; the overflowed
  // orientations are re-run by the ladder as usual).  Returns true when the
  // configuration changed.
  // A batch where most orientations passed the 63-pixel cap in some column
  // switches the rest of the sweep to the priority-carrying strips
  // (configuration 4), which resolve those columns in one pass.
  int adapt_after(int first, int nb, int* c, bool* changed)
  {
    *changed = false;
    static const int kBudgets[] = {73728, 101376, 150528, 0};   // 0: everything the SM allows
    int next = -1;
    if (*c == 0) {
      const size_t cur = cfg[0].smem;
      for (int b : kBudgets) {
        const size_t lim = b ? (size_t)b : (size_t)std::min<size_t>(smem_optin, 227 * 1024) - 2048;
        if (lim > cur + 4096) { next = b ? b : (int)lim; break; }
      }
    }
    if (*c != 0) return 0;
    std::vector<int> fl(nb);
    TOMO_CUDA(cudaStreamSynchronize(side));
    TOMO_CUDA(cudaMemcpy(fl.data(), o_flags.ptr + first, sizeof(int) * nb, cudaMemcpyDeviceToHost));
    int over = 0, cap = 0;
    for (int f : fl) { over += (f & kFlagOverflow) ? 1 : 0; cap += (f & kFlagCap) ? 1 : 0; }
    if (cap * 2 > nb) {
      *c = 4;
      adapt_cfg = 4;
    } else if (next >= 0 && over * 5 > nb) {
      force_h = H;
      normal_smem = next;
      plan_strips();
      adapt_smem = normal_smem; adapt_h = force_h;
    } else {
      return 0;
    }
    choose_strips(*c);
    TOMO_TRY(configure());
    *changed = true;
    return 0;
  }

  int sweep_batches(const int* ids, int n, bool adapt)
  {
    int c = (start_cfg == 4 || (adapt && adapt_cfg == 4)) ? 4 : 0;
    choose_strips(c);
    H_sweep = H;
    TOMO_TRY(configure());
    const int Bo = std::min(batch, n);
    const int bin_cap = 4 * P.n_tri + 4096;
    TOMO_TRY(reserve_outputs());
    // Two batches in flight: batch k+1's binning (reset, rotate, bin
    // count / scan / fill) runs on the binning stream into the other
    // PrepSet while batch k's strips run on main; each batch's fold follows
    // on the side stream.  A set is rebinned only after the fold of the
    // batch that last used it.
    const bool pipe = n > Bo;
    TOMO_TRY(reserve_batch(Bo, bin_cap, pipe ? 2 : 1));
    if (ids) TOMO_CUDA(launch_zero_ids(o_nbed.ptr, ids, n, main));
    else TOMO_CUDA(cudaMemsetAsync(o_nbed.ptr, 0, sizeof(int) * nYPR, main));
    if (pipe) {
      TOMO_CUDA(cudaEventRecord(ev_ready, main));
      TOMO_CUDA(cudaStreamWaitEvent(W.binning, ev_ready, 0));
    }
    EngineParams p = base_params(cfg[c].mode);
    int k = 0;
    for (int first = 0; first < n; first += Bo, k++) {
      const int nb = std::min(Bo, n - first);
      const int which = k & 1;
      const int q = pipe ? which : 0;
      cudaStream_t bs = pipe ? W.binning : main;
      if (k >= 2) TOMO_CUDA(cudaStreamWaitEvent(bs, set[which].folded, 0));
      bind_batch(p, nb, bin_cap, which, first, q);
      if (ids) p.ori = ids + first;
      TOMO_CUDA(launch_bin_count(p, bs, &log));
      TOMO_CUDA(launch_fill(p, bs, &log));
      if (pipe) {
        TOMO_CUDA(cudaEventRecord(W.prep[q].ready, bs));
        TOMO_CUDA(cudaStreamWaitEvent(main, W.prep[q].ready, 0));
      }
      TOMO_CUDA(launch_strip_bed(p, main, cfg[c].smem, &log));
      TOMO_CUDA(cudaEventRecord(ev_ready, main));
      TOMO_CUDA(cudaStreamWaitEvent(side, ev_ready, 0));
      TOMO_CUDA(launch_fold(p, side, &log));
      TOMO_CUDA(cudaEventRecord(set[which].folded, side));
      if (adapt && k < 3 && first + nb < n) {
        bool changed = false;
        TOMO_TRY(adapt_after(first, nb, &c, &changed));
        if (changed) p = base_params(cfg[c].mode);
      }
    }
    // join the side stream back into main
    TOMO_CUDA(cudaEventRecord(ev_ready, side));
    TOMO_CUDA(cudaStreamWaitEvent(main, ev_ready, 0));
    return 0;
  }

  // Re-run a list of orientation ids in configuration c (host-synchronous).
  int run_subset(const std::vector<int>& ids, int c)
  {
    if (ids.empty()) return 0;
    choose_strips(c);
    const int mode = cfg[c].mode;
    TOMO_TRY(configure());
    TOMO_TRY(reserve_outputs());
    TOMO_CUDA(cudaStreamSynchronize(side));
    DevBuf<int> sub;
    TOMO_CUDA(sub.reserve(ids.size()));
    TOMO_CUDA(cudaMemcpyAsync(sub.ptr, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice, main));
    const int Bo = std::min<int>(batch, (int)ids.size());
    const int normal_cap = 4 * P.n_tri + 4096;
    TOMO_TRY(reserve_batch(Bo, mode != 1 ? normal_cap : 1));
    EngineParams p = base_params(mode);
    p.variant = c;
    for (int first = 0; first < (int)ids.size(); first += Bo) {
      const int nb = std::min<int>(Bo, (int)ids.size() - first);
      for (int o = 0; o < nb; o++) TOMO_CUDA(cudaMemsetAsync(o_nbed.ptr + ids[first + o], 0, sizeof(int), main));
      if (mode != 1) {
        bind_batch(p, nb, normal_cap, 0, 0);
        p.ori = sub.ptr + first;
        TOMO_CUDA(launch_batch(p, main, cfg[c].smem, &log));
      } else {
        // the count pass decides the bin capacity, so it runs without one
        bind_batch(p, nb, INT_MAX, 0, 0);
        p.ori = sub.ptr + first;
        TOMO_CUDA(launch_bin_count(p, main, &log));
        std::vector<int> off((size_t)nb * (S + 1));
        TOMO_CUDA(cudaMemcpyAsync(off.data(), bin_off.ptr, sizeof(int) * off.size(), cudaMemcpyDeviceToHost, main));
        TOMO_CUDA(cudaStreamSynchronize(main));
        int cap = 1;
        for (int o = 0; o < nb; o++) cap = std::max(cap, off[(size_t)o * (S + 1) + S]);
        TOMO_CUDA(bins.reserve((size_t)nb * cap));
        p.bins = bins.ptr; p.bin_cap = cap;
        TOMO_CUDA(launch_after_count(p, main, cfg[c].smem, &log));
      }
      TOMO_CUDA(launch_fold(p, main, &log));
    }
    TOMO_CUDA(cudaStreamSynchronize(main));
    sub.release();
    n_redo[c] += (int)ids.size();
    return 0;
  }

  // Per-orientation outputs to the host: all of them, or (after resolve has
  // uploaded a subset to sub_ids) only the subset's, gathered on the device.
  int fetch()
  {
    if (sub_n > 0) return fetch_subset();
    const size_t n = (size_t)nYPR;
    vo64.assign(n, 0); vss64.assign(n, 0); vtc64.assign(n, 0); entries.assign(n, 0); columns.assign(n, 0);
    vof.assign(n, 0.f); vssf.assign(n, 0.f); vtcf.assign(n, 0.f); nbed.assign(n, 0); flags.assign(n, 0);
    if (n == 0 || P.n_tri == 0) return 0;
    TOMO_CUDA(cudaMemcpyAsync(vo64.data(), o_vo.ptr, sizeof(long long) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(vss64.data(), o_vss.ptr, sizeof(long long) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(vtc64.data(), o_vtc.ptr, sizeof(long long) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(entries.data(), o_ent.ptr, sizeof(long long) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(columns.data(), o_col.ptr, sizeof(long long) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(vof.data(), o_vof.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(vssf.data(), o_vssf.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(vtcf.data(), o_vtcf.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(nbed.data(), o_nbed.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaMemcpyAsync(flags.data(), o_flags.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    TOMO_CUDA(cudaStreamSynchronize(side));
    log.collect();
    return 0;
  }

  int fetch_subset()
  {
    const size_t n = (size_t)nYPR, k = (size_t)sub_n;
    if (vo64.size() != n) {
      vo64.assign(n, 0); vss64.assign(n, 0); vtc64.assign(n, 0); entries.assign(n, 0); columns.assign(n, 0);
      vof.assign(n, 0.f); vssf.assign(n, 0.f); vtcf.assign(n, 0.f); nbed.assign(n, 0); flags.assign(n, 0);
    }
    if (P.n_tri == 0) return 0;
    TOMO_CUDA(sub_stage.reserve(k * 10));
    TOMO_CUDA(launch_gather_outputs(o_vo.ptr, o_vss.ptr, o_vtc.ptr, o_ent.ptr, o_col.ptr, o_vof.ptr, o_vssf.ptr,
                                    o_vtcf.ptr, o_nbed.ptr, o_flags.ptr, sub_ids.ptr, sub_n, sub_stage.ptr, main));
    std::vector<long long> h(k * 10);
    TOMO_CUDA(cudaMemcpyAsync(h.data(), sub_stage.ptr, sizeof(long long) * h.size(), cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    TOMO_CUDA(cudaStreamSynchronize(side));
    auto f = [](long long b) { const int i = (int)b; float x; std::memcpy(&x, &i, sizeof(x)); return x; };
    for (size_t q = 0; q < k; q++) {
      const int id = sub_host[q];
      const long long* r = &h[q * 10];
      vo64[id] = r[0]; vss64[id] = r[1]; vtc64[id] = r[2]; entries[id] = r[3]; columns[id] = r[4];
      vof[id] = f(r[5]); vssf[id] = f(r[6]); vtcf[id] = f(r[7]); nbed[id] = (int)r[8]; flags[id] = (int)r[9];
    }
    log.collect();
    return 0;
  }

  // Rotation matrices computed on the host and uploaded only for the listed
  // orientations (uploads made with lazy rotations).
  int ensure_rot(const std::vector<int>& ids)
  {
    std::vector<int> need;
    std::vector<float> compact;
    for (int id : ids) {
      if (rot_ready[id]) continue;
      rotation(h_ypr[id * 3 + 0], h_ypr[id * 3 + 1], h_ypr[id * 3 + 2], &h_rot[(size_t)id * 9]);
      rot_ready[id] = 1;
      need.push_back(id);
      compact.insert(compact.end(), &h_rot[(size_t)id * 9], &h_rot[(size_t)id * 9] + 9);
    }
    if (need.empty()) return 0;
    DevBuf<int> di;
    DevBuf<float> dc;
    TOMO_CUDA(di.reserve(need.size()));
    TOMO_CUDA(dc.reserve(compact.size()));
    TOMO_CUDA(cudaMemcpyAsync(di.ptr, need.data(), sizeof(int) * need.size(), cudaMemcpyHostToDevice, main));
    TOMO_CUDA(cudaMemcpyAsync(dc.ptr, compact.data(), sizeof(float) * compact.size(), cudaMemcpyHostToDevice, main));
    TOMO_CUDA(launch_scatter_rot(rot.ptr, dc.ptr, di.ptr, (int)need.size(), main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    di.release();
    dc.release();
    return 0;
  }

  // Full device phase: the sweep in configuration 0, then the re-runs of
  // flagged orientations: overflowed strip lists in configuration 2, stray
  // hits and priority-dependent columns in configuration 1, and what still
  // overflows in configuration 3.
  int execute()
  {
    if (!force_safe) TOMO_TRY(sweep_device());
    return resolve();
  }

  // After sweep_device: fetch the results and re-run what was flagged.
  // With `subset`, only those orientations were swept and are checked.
  int resolve(const std::vector<int>* subset = nullptr)
  {
    for (int& r : n_redo) r = 0;
    std::vector<int> all;
    sub_n = 0;
    if (!subset) {
      all.resize(nYPR);
      for (int i = 0; i < nYPR; i++) all[i] = i;
      subset = &all;
    } else if (!subset->empty()) {
      TOMO_CUDA(sub_ids.reserve(subset->size()));
      TOMO_CUDA(cudaMemcpyAsync(sub_ids.ptr, subset->data(), sizeof(int) * subset->size(), cudaMemcpyHostToDevice, main));
      sub_host = *subset;
      sub_n = (int)subset->size();
    }
    const int rc = resolve_ids(*subset);
    sub_n = 0;
    return rc;
  }

  int resolve_ids(const std::vector<int>& ids)
  {
    const std::vector<int>* subset = &ids;
    std::vector<int> big, prio, safe, narrow;
    if (force_safe) {
      if (nYPR == 0 || P.n_tri == 0) return fetch();
      TOMO_TRY(reserve_outputs());
      safe = *subset;
    } else {
      TOMO_TRY(fetch());
      for (int i : *subset) {
        if (flags[i] & kFlagGrid) return set_error(TOMO_ERR_CAPACITY, "slot index outside the grid");
        if (flags[i] & (kFlagStray | kFlagBinCap)) safe.push_back(i);
        else if (flags[i] & kFlagOverflow) big.push_back(i);
        else if (flags[i] & kFlagCap) prio.push_back(i);
      }
      if (!big.empty()) {
        TOMO_TRY(run_subset(big, 2));
        TOMO_TRY(fetch());
        for (int id : big) {
          if (flags[id] & (kFlagStray | kFlagBinCap | kFlagOverflow)) safe.push_back(id);
          else if (flags[id] & kFlagCap) prio.push_back(id);
        }
      }
      if (!prio.empty()) {
        TOMO_TRY(run_subset(prio, 4));
        TOMO_TRY(fetch());
        for (int id : prio)
          if (flags[id] & kFlagRedo) safe.push_back(id);
      }
    }
    if (!safe.empty()) {
      TOMO_TRY(run_subset(safe, 1));
      TOMO_TRY(fetch());
      for (int id : safe)
        if (flags[id] & kFlagSafeOverflow) narrow.push_back(id);
    }
    if (!narrow.empty()) {
      TOMO_TRY(run_subset(narrow, 3));
      TOMO_TRY(fetch());
    }
    for (int i : *subset) {
      if (flags[i] & kFlagSafeOverflow) return set_error(TOMO_ERR_CAPACITY, "column strip exceeds shared memory");
      if (flags[i] & kFlagGrid) return set_error(TOMO_ERR_CAPACITY, "slot index outside the grid");
      if (flags[i] & kFlagRedo) return set_error(TOMO_ERR_CAPACITY, "orientation unresolved after the re-runs");
      if (flags[i] & kFlagFoldRange)
        return set_error(TOMO_ERR_CAPACITY, "column values past 16 bits overflowed the fold escape table");
    }
    n_safe = n_redo[1] + n_redo[2] + n_redo[3] + n_redo[4];
    return 0;
  }

  // One orientation with the dense per-column dump enabled (parity tests).
  int dump(int id, int c, int* cols8, unsigned* keys64, short* types64)
  {
    const int fl = dump_device(id, c);
    if (fl < 0) return fl;
    const size_t GG = (size_t)G * G;
    if (cols8) TOMO_CUDA(cudaMemcpyAsync(cols8, dump_cols.ptr, sizeof(int) * GG * 8, cudaMemcpyDeviceToHost, main));
    if (keys64) TOMO_CUDA(cudaMemcpyAsync(keys64, dump_keys.ptr, sizeof(unsigned) * GG * 64, cudaMemcpyDeviceToHost, main));
    if (types64) TOMO_CUDA(cudaMemcpyAsync(types64, dump_types.ptr, sizeof(short) * GG * 64, cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    return fl;
  }

  // The same dump compacted on the device to the occupied columns:
  // cols9[n_occ][9] = slot id + the 8 dump fields, keys/types = each occupied
  // column's kept keys and types, concatenated in slot order.
  int dump_compact(int id, int c, std::vector<int>& cols9, std::vector<unsigned>& keys, std::vector<short>& types)
  {
    const int fl = dump_device(id, c);
    if (fl < 0) return fl;
    const int GG = G * G;
    TOMO_CUDA(dump_off.reserve((size_t)GG * 2));
    TOMO_CUDA(dump_tot.reserve(2));
    TOMO_CUDA(launch_dump_scan(dump_cols.ptr, GG, dump_off.ptr, dump_tot.ptr, main));
    int tot[2] = {0, 0};
    TOMO_CUDA(cudaMemcpyAsync(tot, dump_tot.ptr, sizeof(tot), cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    TOMO_CUDA(dump_ccols.reserve((size_t)tot[0] * 9));
    TOMO_CUDA(dump_ckeys.reserve((size_t)tot[1]));
    TOMO_CUDA(dump_ctypes.reserve((size_t)tot[1]));
    TOMO_CUDA(launch_dump_gather(dump_cols.ptr, dump_keys.ptr, dump_types.ptr, GG, dump_off.ptr, dump_ccols.ptr,
                                 dump_ckeys.ptr, dump_ctypes.ptr, main));
    cols9.resize((size_t)tot[0] * 9);
    keys.resize((size_t)tot[1]);
    types.resize((size_t)tot[1]);
    if (tot[0]) TOMO_CUDA(cudaMemcpyAsync(cols9.data(), dump_ccols.ptr, sizeof(int) * cols9.size(), cudaMemcpyDeviceToHost, main));
    if (tot[1]) {
      TOMO_CUDA(cudaMemcpyAsync(keys.data(), dump_ckeys.ptr, sizeof(unsigned) * keys.size(), cudaMemcpyDeviceToHost, main));
      TOMO_CUDA(cudaMemcpyAsync(types.data(), dump_ctypes.ptr, sizeof(short) * types.size(), cudaMemcpyDeviceToHost, main));
    }
    TOMO_CUDA(cudaStreamSynchronize(main));
    return fl;
  }

  // Runs one orientation in strip configuration c with the dense dump on;
  // returns its status flags.
  int dump_device(int id, int c)
  {
    if (id < 0 || id >= nYPR) return set_error(TOMO_ERR_ARG, "orientation index out of range");
    if (P.n_tri == 0) return set_error(TOMO_ERR_ARG, "empty mesh");
    if (c < 0 || c > 4) return set_error(TOMO_ERR_ARG, "bad strip configuration");
    choose_strips(c);
    const int mode = cfg[c].mode;
    const size_t smem = cfg[c].smem;
    TOMO_TRY(configure());
    TOMO_TRY(reserve_outputs());
    const size_t GG = (size_t)G * G;
    TOMO_CUDA(dump_cols.reserve(GG * 8)); TOMO_CUDA(dump_keys.reserve(GG * 64)); TOMO_CUDA(dump_types.reserve(GG * 64));
    TOMO_CUDA(cudaMemsetAsync(dump_cols.ptr, 0, sizeof(int) * GG * 8, main));
    TOMO_CUDA(cudaMemsetAsync(dump_keys.ptr, 0, sizeof(unsigned) * GG * 64, main));
    TOMO_CUDA(cudaMemsetAsync(dump_types.ptr, 0, sizeof(short) * GG * 64, main));
    TOMO_CUDA(cudaMemsetAsync(o_nbed.ptr + id, 0, sizeof(int), main));
    EngineParams p = base_params(mode);
    p.dump_slot = 0; p.dump_cols = dump_cols.ptr; p.dump_keys = dump_keys.ptr; p.dump_types = dump_types.ptr;
    int cap = 4 * P.n_tri + 4096;
    TOMO_TRY(reserve_batch(1, mode != 1 ? cap : 1));
    bind_batch(p, 1, mode != 1 ? cap : INT_MAX, 0, id);
    if (mode != 1) {
      TOMO_CUDA(launch_batch(p, main, smem, &log));
    } else {
      TOMO_CUDA(launch_bin_count(p, main, &log));
      int total = 0;
      TOMO_CUDA(cudaMemcpyAsync(&total, bin_off.ptr + S, sizeof(int), cudaMemcpyDeviceToHost, main));
      TOMO_CUDA(cudaStreamSynchronize(main));
      cap = std::max(total, 1);
      TOMO_CUDA(bins.reserve((size_t)cap));
      p.bins = bins.ptr; p.bin_cap = cap;
      TOMO_CUDA(launch_after_count(p, main, smem, &log));
    }
    TOMO_CUDA(launch_fold(p, main, &log));
    int fl = 0;
    TOMO_CUDA(cudaMemcpyAsync(&fl, o_flags.ptr + id, sizeof(int), cudaMemcpyDeviceToHost, main));
    TOMO_CUDA(cudaStreamSynchronize(main));
    return fl;
  }

  // Autotuner: times the device sweep of an evenly strided sample of up to
  // `sample` orientations for each candidate (orientations per batch,
  // shared-memory budget of a normal strip CTA -- which sets the strip
  // height, the entry capacity and the CTAs per SM) and keeps the fastest.
  // Only the speed depends on the choice: every configuration's results are
  // exact (overflowing strips are re-run).
  // Strip configuration of a sweep picked by the batch autotuner.
  struct TuneResult { int batch, normal_smem, strip_h, start_cfg; double us_per_orientation; };

  // Times candidate configurations on an evenly strided sample of the
  // orientations and keeps the fastest.  A candidate's time covers the whole
  // sweep of the sample, re-runs included: the configuration-0 strips, then
  // the ladder that re-runs what they flagged (Engine::resolve), so a budget
  // too small for the mesh pays for its overflows.  Candidates: 128 or 256
  // orientations per batch x the normal strip budget (four CTAs per SM, 72 KB,
  // 99 KB) x the strip height (the planned one and half of it).  When most of
  // the sample passes the 63-pixel cap in some column, every candidate starts
  // in the priority-carrying strips (configuration 4), as an adaptive sweep
  // would switch to them.
  int autotune(int sample, TuneResult* best)
  {
    static const int kBatches[] = {128, 256};
    static const int kSmem[] = {0, 73728, 101376};   // 0: four CTAs per SM
    best->batch = batch; best->normal_smem = normal_smem; best->strip_h = force_h; best->start_cfg = start_cfg;
    best->us_per_orientation = 0.0;
    if (nYPR == 0 || P.n_tri == 0) return 0;
    const int n = std::min(nYPR, std::max(sample, 1));
    std::vector<int> ids(n);
    for (int i = 0; i < n; i++) ids[i] = (int)((long long)i * nYPR / n);
    DevBuf<int> dids;
    TOMO_CUDA(dids.reserve(n));
    TOMO_CUDA(cudaMemcpyAsync(dids.ptr, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice, main));
    cudaEvent_t a = nullptr, b = nullptr;
    TOMO_CUDA(cudaEventCreate(&a));
    TOMO_CUDA(cudaEventCreate(&b));
    const bool timing = log.timing;
    log.timing = false;
    const int keep_batch = batch, keep_smem = normal_smem, keep_h = force_h, keep_cfg = start_cfg;
    double best_us = 1e300;
    int rc = 0;
    // the planned strip height, and whether the sample is cap-heavy
    plan_strips();
    const int h_plan = cfg[0].H;
    start_cfg = 0;
    if ((rc = sweep_device(dids.ptr, n)) == 0) {
      std::vector<int> fl(nYPR);
      if (cudaStreamSynchronize(side) != cudaSuccess || cudaStreamSynchronize(main) != cudaSuccess ||
          cudaMemcpy(fl.data(), o_flags.ptr, sizeof(int) * nYPR, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = set_error(TOMO_ERR_CUDA, "autotune flags");
      int capped = 0;
      for (int i = 0; rc == 0 && i < n; i++) capped += (fl[ids[i]] & kFlagCap) ? 1 : 0;
      if (rc == 0 && capped * 2 > n) start_cfg = 4;
    }
    const int tuned_cfg = start_cfg;
    for (int bsz : kBatches) {
      if (rc) break;
      for (int sm : kSmem) {
        if (rc) break;
        for (int h : {h_plan, h_plan / 2}) {
          if (h < 1 || (h != h_plan && h_plan < 2)) continue;
          batch = bsz; normal_smem = sm; force_h = (h == h_plan) ? keep_h : h;
          plan_strips();
          if (force_h && cfg[0].H != force_h) continue;   // the budget cannot hold that strip height
          float ms = 0.f;
          // an untimed run first: it allocates and warms
          if ((rc = sweep_device(dids.ptr, n)) != 0) break;
          if ((rc = resolve(&ids)) != 0) break;
          if (cudaEventRecord(a, main) != cudaSuccess) { rc = set_error(TOMO_ERR_CUDA, "autotune event"); break; }
          if ((rc = sweep_device(dids.ptr, n)) != 0) break;
          if ((rc = resolve(&ids)) != 0) break;
          if (cudaEventRecord(b, main) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess ||
              cudaEventElapsedTime(&ms, a, b) != cudaSuccess) { rc = set_error(TOMO_ERR_CUDA, "autotune timing"); break; }
          const double us = 1000.0 * ms / n;
          if (us < best_us) {
            best_us = us; best->batch = bsz; best->normal_smem = sm; best->strip_h = force_h;
            best->start_cfg = tuned_cfg;
          }
        }
      }
    }
    log.timing = timing;
    cudaStreamSynchronize(main);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    dids.release();
    batch = rc ? keep_batch : best->batch;
    normal_smem = rc ? keep_smem : best->normal_smem;
    force_h = rc ? keep_h : best->strip_h;
    start_cfg = rc ? keep_cfg : best->start_cfg;
    plan_strips();
    best->us_per_orientation = best_us;
    return rc;
  }

  // Float fold of n additions of BedThickness: Calculate adds
  // sumType(typeBed) * BedThickness per bed slot (STomoSh_INT3.cpp:1240), and
  // every bed slot holds exactly one bed pixel at z = 1.
  void finalize_host()
  {
    const size_t n = (size_t)nYPR;
    Mo.assign(n + 2, 0.f); Mss.assign(n + 2, 0.f); Vtc.assign(n + 2, 0.f);
    int maxbed = 0;
    for (size_t i = 0; i < n; i++) maxbed = std::max(maxbed, nbed[i]);
    std::vector<float> bedfold((size_t)maxbed + 1, 0.f);
    for (int k = 1; k <= maxbed; k++) bedfold[k] = bedfold[k - 1] + (float)1 * P.bed_thickness;
    for (size_t i = 0; i < n; i++) {
      float vm[22] = {0};
      vm[8] = vof[i];
      vm[4] = vssf[i];
      vm[2] = vtcf[i];
      vm[11] = bedfold[nbed[i]];
      vol_to_mass(P, vm);
      Mo[i] = vm[16];
      Mss[i] = vm[13];
      Vtc[i] = vm[2];
    }
  }
};

namespace {
Engine* g_engine = nullptr;
std::vector<float> g_Mss, g_Mo, g_Vtc;
std::vector<long long> g_Vo64, g_Vss64, g_Vtc64;
float g_volmass[22] = {0};
float g_mat4x4[16] = {0};
std::vector<short> g_pix[11];
int g_npix[11] = {0};

Engine& engine()
{
  if (!g_engine) g_engine = new Engine(*new Workspace(), true);
  return *g_engine;
}

// mat4x4 of STomoSh_Base::Rotate (STomoSh_Base.cpp:155-167) for one orientation.
void host_mat4x4(const Engine& E, const float* vtx, int nV, int id, float* m16)
{
  const float* R = &E.h_rot[(size_t)id * 9];
  float mn[3] = {1e5f, 1e5f, 1e5f};
  for (int v = 0; v < nV; v++) {
    const float t0 = vtx[v * 3 + 0] - E.cx, t1 = vtx[v * 3 + 1] - E.cy, t2 = vtx[v * 3 + 2] - E.cz;
    for (int r = 0; r < 3; r++) {
      float s = R[r * 3 + 0] * t0;
      s += R[r * 3 + 1] * t1;
      s += R[r * 3 + 2] * t2;
      s += 0.0f * 1.0f;
      mn[r] = (mn[r] <= s) ? mn[r] : s;
    }
  }
  const float dx = mn[0] - E.P.bed_outer, dy = mn[1] - E.P.bed_outer, dz = mn[2];
  const float m = -E.cx, n = -E.cy, o = -E.cz;
  std::memset(m16, 0, 16 * sizeof(float));
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < 3; k++) m16[r * 4 + k] = R[r * 3 + k];
  m16[15] = 1.f;
  m16[3] = -dx + R[0] * m + R[1] * n + R[2] * o;
  m16[7] = -dy + R[3] * m + R[4] * n + R[5] * o;
  m16[11] = -dz + R[6] * m + R[7] * n + R[8] * o;
}
// Final slot rows of one orientation rebuilt on the host from its column
// dump: kept pixels in column order with their paired types, the floor
// sentinels (STomoSh_INT3.cpp:790-810) and the bed pixels (GenerateBed,
// :1375-1443) -- the reference's slot buffer after thread_func.  From them:
// the render pixels of slotsToPxls (:1103-1135) and GetSSPixels
// (:1257-1318, brief branch) and the vm_info of Calculate (:1211-1255).
struct SlotRow { short type, z, nz; };

bool host_bed_candidate(const Engine& E, const std::vector<uint8_t>& bf, int X, int Y)
{
  const int G = E.G, r = (int)E.P.bed_outer;
  const int xa = std::max(X - r, 0), xb = std::min(X + r, G), ya = std::max(Y - r, 0), yb = std::min(Y + r, G);
  const int qid = X * G + Y;
  float md = 1e5f;
  for (int sx = xa; sx < xb; sx++)
    for (int sy = ya; sy < yb; sy++) {
      const int sid = sx * G + sy;
      const uint8_t f = bf[sid];
      if (!(f & kBfTouch)) continue;
      if ((f & kBfSelfR) && sid < qid) continue;
      const float dx = (float)X - (float)sx, dy = (float)Y - (float)sy;
      const float dist = sqrtf(dx * dx + dy * dy);
      md = (md < dist) ? md : dist;
    }
  if (md > E.P.bed_outer) return false;
  if (E.P.bed_type == kBedBrim || E.P.bed_type == kBedRaft) return true;
  if (E.P.bed_type == kBedSkirt && md > E.P.bed_inner) return true;
  return false;
}

int export_best(Engine& E, int id, std::vector<short>* pix, int* npix, float* vm)
{
  const int G = E.G;
  const size_t GG = (size_t)G * G;
  std::vector<int> cols;
  std::vector<unsigned> keys;
  std::vector<short> types;
  int fl = -1;
  for (int c : {0, 4, 1, 3}) {
    fl = E.dump_compact(id, c, cols, keys, types);
    if (fl < 0) return fl;
    if (!(fl & (kFlagRedo | kFlagSafeOverflow))) break;
  }
  if (fl & (kFlagRedo | kFlagSafeOverflow | kFlagGrid))
    return set_error(TOMO_ERR_CAPACITY, "best orientation could not be exported");
  // occupied columns in slot order: rows[rbeg[j] .. rbeg[j+1]) plus an
  // optional bed row (bed_row[j]); bed-only columns listed separately
  const int nocc = (int)(cols.size() / 9);
  std::vector<SlotRow> rows;
  rows.reserve(keys.size() + 2 * (size_t)nocc);
  std::vector<int> rbeg((size_t)nocc + 1, 0);
  std::vector<int> colidx(GG, -1);
  std::vector<uint8_t> bed_row((size_t)nocc, 0);
  std::vector<uint8_t> bf(GG, (uint8_t)(kBfPoss | kBfLand));
  int minX = G, minY = G, maxX = -1, maxY = -1;
  size_t k0 = 0;
  for (int j = 0; j < nocc; j++) {
    const int* c = &cols[(size_t)j * 9];
    const int sl = c[0], nd = c[1], nfin = c[2];
    const int x = sl / G, y = sl % G;
    minX = std::min(minX, x); maxX = std::max(maxX, x); minY = std::min(minY, y); maxY = std::max(maxY, y);
    rbeg[j] = (int)rows.size();
    const int n = std::min(nd, 64);
    for (int i = 0; i < n; i++) {
      const unsigned k = keys[k0 + i];
      rows.push_back({nd > 1 ? types[k0 + i] : (short)0, (short)((int)(k >> 16) - 32768), (short)((int)(k & 0xFFFFu) - 32768)});
    }
    k0 += (size_t)n;
    const int extra = nfin - nd;
    if (extra == 2) { rows.push_back({(short)kSSA, 0, 0}); rows.push_back({(short)kNVA, 0, 0}); }
    else if (extra == 1) rows.push_back({(short)c[7], 0, 0});
    bf[sl] = (uint8_t)c[8];
    colidx[sl] = j;
  }
  rbeg[nocc] = (int)rows.size();
  // bed pixels, in the reference's scan order
  std::vector<int> bed_only;
  if (E.P.bed_type != kBedNone && maxX >= 0 && (int)E.P.bed_outer > 0) {
    const int m = (int)E.P.bed_outer + 1;
    const int bx0 = std::max(minX - m, 0), bx1 = std::min(maxX + m + 1, G);
    const int by0 = std::max(minY - m, 0), by1 = std::min(maxY + m + 1, G);
    for (int X = bx0; X < bx1; X++)
      for (int Y = by0; Y < by1; Y++) {
        const size_t sl = (size_t)X * G + Y;
        const uint8_t f = bf[sl];
        if (!((f & kBfPoss) && (f & kBfLand)) || !host_bed_candidate(E, bf, X, Y)) continue;
        const int j = colidx[sl];
        if (j < 0) { bed_only.push_back((int)sl); continue; }
        bool merged = false;
        for (int r = rbeg[j]; r < rbeg[j + 1]; r++)
          if (rows[r].z == 1 && rows[r].nz == 0) { rows[r].type |= (short)kBed; merged = true; break; }
        if (!merged) bed_row[j] = 1;
      }
  }
  // render pixels per type (slotsToPxls), the support pixels (GetSSPixels)
  // and the float folds of Calculate, over the final slots in ascending order
  for (int k = 0; k < 11; k++) pix[k].clear();
  float va = 0.f, vb = 0.f, vnv = 0.f, vtc = 0.f, vbed = 0.f;
  const SlotRow bed_px = {(short)kBed, 1, 0};
  auto column = [&](int sl, const SlotRow* r, int n, bool extra_bed) {
    const short x = (short)(sl / G), y = (short)(sl % G);
    int sa = 0, sb = 0, snvb = 0, snva = 0, stc = 0, sbed = 0;
    int ss0 = -1, ss1 = -1;
    for (int i = 0; i < n + (extra_bed ? 1 : 0); i++) {
      const SlotRow& q = i < n ? r[i] : bed_px;
      for (int k = 0; k < 11; k++)
        if (k != 4 && (q.type & (1 << k))) {
          const short px[6] = {x, y, q.z, 0, 0, q.nz};
          pix[k].insert(pix[k].end(), px, px + 6);
        }
      if (q.type & kSSB) ss0 = q.z;
      if (q.type & kSSA) ss1 = q.z;
      if (ss0 > -1 && ss1 > -1) {
        for (int zz = ss0; zz >= ss1; zz--) {
          const short px[6] = {x, y, (short)zz, 0, 0, 0};
          pix[4].insert(pix[4].end(), px, px + 6);
        }
        ss0 = ss1 = -1;
      }
      if (q.type & kAl) sa += q.z;
      if (q.type & kBe) sb += q.z;
      if (q.type & kNVB) snvb += q.z;
      if (q.type & kNVA) snva += q.z;
      if (q.type & kTC) stc += q.z;
      if (q.type & kBed) sbed += q.z;
    }
    va += (float)sa; vb += (float)sb; vnv += (float)(snvb - snva); vtc += (float)stc;
    vbed += (float)sbed * E.P.bed_thickness;
  };
  size_t b = 0;
  for (int j = 0; j <= nocc; j++) {
    const int sl = j < nocc ? cols[(size_t)j * 9] : INT_MAX;
    while (b < bed_only.size() && bed_only[b] < sl) { column(bed_only[b], nullptr, 0, true); b++; }
    if (j < nocc) column(sl, rows.data() + rbeg[j], rbeg[j + 1] - rbeg[j], bed_row[j] != 0);
  }
  for (int k = 0; k < 11; k++) npix[k] = (int)(pix[k].size() / 6);
  vm[0] = va; vm[1] = vb; vm[2] = vtc; vm[3] = vnv; vm[11] = vbed;
  return 0;
}

}  // namespace

}  // namespace tomo

using namespace tomo;

// ------------------------------------------------ C-ABI

extern "C" {

int TomoSh_CUDA(float* f32info, int* i32info, float* YPR, int* tri, float* vtx, float* vtx_nrm, float* tri_nrm,
                int* chull_tri, float* chull_vtx, float* chull_trinrm)
{
  (void)tri_nrm; (void)chull_tri; (void)chull_vtx; (void)chull_trinrm;
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  if (f32info == nullptr || i32info == nullptr) return set_error(TOMO_ERR_ARG, "info arrays are null");
  Engine& E = engine();
  int rc = E.init();
  if (rc) return rc;
  rc = E.upload(f32info, i32info, YPR, tri, vtx, vtx_nrm);
  if (rc) return rc;
  rc = E.execute();
  if (rc) return rc;
  E.finalize_host();
  const int n = E.nYPR;
  g_Mss.assign(E.Mss.begin(), E.Mss.end());
  g_Mo.assign(E.Mo.begin(), E.Mo.end());
  g_Vtc.assign(E.Vtc.begin(), E.Vtc.end());
  g_Vo64 = E.vo64; g_Vss64 = E.vss64; g_Vtc64 = E.vtc64;
  const int opt = first_optimal(n, g_Mss.data());
  std::memset(g_volmass, 0, sizeof(g_volmass));
  for (int k = 0; k < 11; k++) { g_pix[k].clear(); g_npix[k] = 0; }
  if (n > 0) {
    if (E.P.n_tri > 0 && E.export_pixels) {
      rc = export_best(E, opt, g_pix, g_npix, g_volmass);
      if (rc) return rc;
    } else {
      g_volmass[2] = E.vtcf[opt];
    }
    g_volmass[8] = E.vof[opt]; g_volmass[4] = E.vssf[opt];
    vol_to_mass(E.P, g_volmass);
    host_mat4x4(E, vtx, E.P.n_vtx, opt, g_mat4x4);
  }
  return opt;
}

// The reference exports the CPU engine under this name (Tomo_Shell2026.cpp:257-260);
// here it is the same B200 computation, whose results are the INT3 results.
int TomoSh_INT3(float* f32info, int* i32info, float* YPR, int* tri, float* vtx, float* vtx_nrm, float* tri_nrm,
                int* chull_tri, float* chull_vtx, float* chull_trinrm)
{
  return TomoSh_CUDA(f32info, i32info, YPR, tri, vtx, vtx_nrm, tri_nrm, chull_tri, chull_vtx, chull_trinrm);
}

float* getMss(void) { return g_Mss.empty() ? nullptr : g_Mss.data(); }
float* getMo(void) { return g_Mo.empty() ? nullptr : g_Mo.data(); }
float* getVtc(void) { return g_Vtc.empty() ? nullptr : g_Vtc.data(); }
float* getVolMassInfo(void) { return g_volmass; }
float* getMat4x4(void) { return g_mat4x4; }
int getnData2i(short type) { return (type >= 0 && type < 11) ? g_npix[type] : 0; }
short* getpData2i(short type)
{
  if (type < 0 || type >= 11 || g_pix[type].empty()) return nullptr;
  return g_pix[type].data();
}
const long long* getVo64(void) { return g_Vo64.empty() ? nullptr : g_Vo64.data(); }
const long long* getVss64(void) { return g_Vss64.empty() ? nullptr : g_Vss64.data(); }
const long long* getVtc64(void) { return g_Vtc64.empty() ? nullptr : g_Vtc64.data(); }

void OnDestroy(void)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_Mss.clear(); g_Mo.clear(); g_Vtc.clear(); g_Vo64.clear(); g_Vss64.clear(); g_Vtc64.clear();
  g_Mss.shrink_to_fit(); g_Mo.shrink_to_fit(); g_Vtc.shrink_to_fit();
  for (auto& v : g_pix) { v.clear(); v.shrink_to_fit(); }
  std::memset(g_npix, 0, sizeof(g_npix));
  if (g_engine) {
    Workspace* w = &g_engine->W;
    g_engine->release();
    delete g_engine;
    delete w;
    g_engine = nullptr;
  }
}

int tomoGetLastError(void) { return g_last_error; }
const char* tomoGetLastErrorString(void) { return g_last_error_str.c_str(); }

void tomoRotation(float yaw, float pitch, float roll, float* out9) { rotation(yaw, pitch, roll, out9); }

float tomoShadowThreshold(float theta_c) { return (float)(-1.0 * (double)sinf(theta_c)); }

void tomoVolToMass(const float* f32info, const int* i32info, float* vm22)
{
  vol_to_mass(read_params(f32info, i32info), vm22);
}

int tomoSetOption(int key, int value)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  Engine& E = engine();
  switch (key) {
    case TOMO_OPT_BATCH: if (value < 1) return TOMO_ERR_ARG; E.batch = value; return 0;
    case TOMO_OPT_STRIP_H: if (value < 0 || value > 8) return TOMO_ERR_ARG; E.force_h = value; return 0;
    case TOMO_OPT_FORCE_SAFE: E.force_safe = value ? 1 : 0; return 0;
    case TOMO_OPT_NORMAL_SMEM: if (value < 0 || value > 232448) return TOMO_ERR_ARG; E.normal_smem = value; return 0;
    case TOMO_OPT_EXPORT: E.export_pixels = value ? 1 : 0; return 0;
    case TOMO_OPT_ADAPTIVE: E.adaptive = value ? 1 : 0; E.adapt_smem = E.adapt_h = E.adapt_cfg = 0; return 0;
    case TOMO_OPT_PROPOSAL: if (value < 0 || value > 2) return TOMO_ERR_ARG; g_proposal = value; return 0;
    case TOMO_OPT_FOLD_LIMIT: if (value < 1 || value > 32767) return TOMO_ERR_ARG; E.fold_lim = value; return 0;
    default: return TOMO_ERR_ARG;
  }
}

int tomoGetStats(long long* out, int n)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (out == nullptr) return TOMO_ERR_ARG;
  long long v[12] = {0};
  if (g_engine) {
    const Engine& E = *g_engine;
    const long long e[9] = {E.G, E.H_sweep, (E.G + std::max(E.H_sweep, 1) - 1) / std::max(E.H_sweep, 1),
                            E.cfg[0].C, E.n_redo[2], E.nYPR, E.batch, E.n_redo[1] + E.n_redo[3], E.n_redo[4]};
    for (int i = 0; i < 9; i++) v[i] = e[i];
  }
  v[9] = g_static_reruns[2];
  v[10] = g_static_reruns[4];
  v[11] = g_static_reruns[1] + g_static_reruns[3];
  for (int i = 0; i < n && i < 12; i++) out[i] = v[i];
  return 0;
}

// Per-orientation exact results of the last TomoSh_CUDA / tomoSweep call.
int tomoGetResults(long long* vo64, long long* vss64, long long* vtc64, float* vof, float* vssf, float* vtcf,
                   int* nbed, int* flags, long long* entries, long long* columns)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_engine) return TOMO_ERR_ARG;
  const Engine& E = *g_engine;
  const size_t n = (size_t)E.nYPR;
  if (vo64) std::memcpy(vo64, E.vo64.data(), sizeof(long long) * n);
  if (vss64) std::memcpy(vss64, E.vss64.data(), sizeof(long long) * n);
  if (vtc64) std::memcpy(vtc64, E.vtc64.data(), sizeof(long long) * n);
  if (vof) std::memcpy(vof, E.vof.data(), sizeof(float) * n);
  if (vssf) std::memcpy(vssf, E.vssf.data(), sizeof(float) * n);
  if (vtcf) std::memcpy(vtcf, E.vtcf.data(), sizeof(float) * n);
  if (nbed) std::memcpy(nbed, E.nbed.data(), sizeof(int) * n);
  if (flags) std::memcpy(flags, E.flags.data(), sizeof(int) * n);
  if (entries) std::memcpy(entries, E.entries.data(), sizeof(long long) * n);
  if (columns) std::memcpy(columns, E.columns.data(), sizeof(long long) * n);
  return 0;
}

// Split entry points: upload once, run the device sweep repeatedly (inputs
// resident in HBM), then fetch.  The sweep runs on the engine's own streams;
// tomoSweepDevice records cudaEvents around its work when given non-null
// events (created by the caller) and returns after the device finished.
int tomoPrepare(const float* f32info, const int* i32info, const float* YPR, const int* tri, const float* vtx,
                const float* vtx_nrm)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  Engine& E = engine();
  int rc = E.init();
  if (rc) return rc;
  return E.upload(f32info, i32info, YPR, tri, vtx, vtx_nrm);
}

int tomoSweepDevice(void* ev_start, void* ev_stop, float* kernel_ms)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_engine || !g_engine->main) return set_error(TOMO_ERR_ARG, "tomoPrepare was not called");
  Engine& E = *g_engine;
  cudaEvent_t a = (cudaEvent_t)ev_start, b = (cudaEvent_t)ev_stop;
  cudaEvent_t la = nullptr, lb = nullptr;
  if (!a) { TOMO_CUDA(cudaEventCreate(&la)); a = la; }
  if (!b) { TOMO_CUDA(cudaEventCreate(&lb)); b = lb; }
  TOMO_CUDA(cudaEventRecord(a, E.main));
  int rc = E.execute();
  if (rc == 0) {
    TOMO_CUDA(cudaEventRecord(b, E.main));
    TOMO_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    TOMO_CUDA(cudaEventElapsedTime(&ms, a, b));
    E.last_kernel_ms = ms;
    if (kernel_ms) *kernel_ms = ms;
  }
  if (la) cudaEventDestroy(la);
  if (lb) cudaEventDestroy(lb);
  return rc;
}

int tomoProfile(int enable, int reset)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  Engine& E = engine();
  if (reset) E.log.reset();
  E.log.timing = enable != 0;
  return 0;
}

int tomoGetKernelLog(long long* launches, double* ms, long long* timed, int n)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_engine) return TOMO_ERR_ARG;
  const LaunchLog& L = g_engine->log;
  for (int k = 0; k < n && k < kKinds; k++) {
    if (launches) launches[k] = L.launches[k];
    if (ms) ms[k] = L.ms[k];
    if (timed) timed[k] = L.timed[k];
  }
  return kKinds;
}

int tomoProbeReadBandwidth(const void* dev_buf, long long bytes, int reps, float* ms_out)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!dev_buf || bytes < 16 || (reinterpret_cast<uintptr_t>(dev_buf) & 15) != 0 || reps <= 0 || !ms_out)
    return set_error(TOMO_ERR_ARG, "read probe: need a 16-byte aligned device buffer of at least 16 bytes");
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, dev_buf) != cudaSuccess || pa.type != cudaMemoryTypeDevice)
    return set_error(TOMO_ERR_ARG, "read probe: the buffer is not device memory");
  int dev = 0, sms = 0;
  TOMO_CUDA(cudaGetDevice(&dev));
  TOMO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaStream_t s = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = 0;
  float ms = 0.f;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&a) != cudaSuccess ||
      cudaEventCreate(&b) != cudaSuccess)
    rc = set_error(TOMO_ERR_CUDA, "read probe: stream or event creation failed");
  // one untimed pass brings the buffer into L2 when it fits
  else if (launch_read_probe(dev_buf, bytes, 1, 8 * sms, s) != cudaSuccess || cudaEventRecord(a, s) != cudaSuccess ||
           launch_read_probe(dev_buf, bytes, reps, 8 * sms, s) != cudaSuccess || cudaEventRecord(b, s) != cudaSuccess ||
           cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess)
    rc = set_error(TOMO_ERR_CUDA, "read probe: launch or timing failed");
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (s) cudaStreamDestroy(s);
  if (rc == 0) *ms_out = ms;
  return rc;
}

int tomoGridSize(void)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_engine ? g_engine->G : 0;
}

int tomoColumnDump(int ypr_index, int safe_mode, int* cols8, unsigned* keys64, short* types64)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_engine || !g_engine->main) return set_error(TOMO_ERR_ARG, "tomoPrepare was not called");
  return g_engine->dump(ypr_index, safe_mode ? 1 : 0, cols8, keys64, types64);
}

int tomoFinish(float* Mo, float* Mss, float* Vtc)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_engine) return set_error(TOMO_ERR_ARG, "tomoPrepare was not called");
  Engine& E = *g_engine;
  E.finalize_host();
  const size_t n = (size_t)E.nYPR;
  if (Mo) std::memcpy(Mo, E.Mo.data(), sizeof(float) * n);
  if (Mss) std::memcpy(Mss, E.Mss.data(), sizeof(float) * n);
  if (Vtc) std::memcpy(Vtc, E.Vtc.data(), sizeof(float) * n);
  return first_optimal((int)n, E.Mss.data());
}

}  // extern "C"

// ------------------------------------------------ allocation-free sweep
//
// tomoSweepStatic: the orientation search of TomoSh_CUDA for small meshes,
// with every device buffer carved out of one file-scope __device__ array
// and every host buffer a file-scope array, so that a call allocates no
// memory on the device or the host.  The kernels, the strip configurations
// and the re-run ladder are those of Engine::resolve_ids (overflow ->
// configuration 2, a column past the 63-pixel cap -> priority strips,
// configuration 4, stray hits or what is still unresolved -> safe mode,
// configuration 1, then one-column safe strips, configuration 3); only the
// buffers and the batch size (kStaticBatch orientations) differ.

namespace tomo {

constexpr size_t kStaticArenaBytes = size_t(8) << 20;   // 8 MiB of device scratch per device
constexpr int kStaticMaxTri = 16384;
constexpr int kStaticMaxVtx = 16384;
constexpr int kStaticBatch = 4;
constexpr int kStaticGrid = 256;                        // the reference's slot grid
constexpr int kStaticMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_arena[kStaticArenaBytes];

namespace {

constexpr size_t static_round(size_t b) { return (b + 255) & ~size_t(255); }

// Bytes of the arena layout below for nV vertices and nT triangles.
constexpr size_t static_bytes(size_t nV, size_t nT)
{
  const size_t B = kStaticBatch, GG = (size_t)kStaticGrid * kStaticGrid, S = kStaticGrid;  // S bound: 1-column strips
  return static_round(16 * nV) * 2 + static_round(16 * nT) + static_round(4 * 9 * B) + static_round(4 * B) +
         static_round(16 * B * nV) + static_round(4 * 4 * B) + static_round(4 * B * nT) +
         static_round(4 * B * (S + 1)) + static_round(4 * B * S) + static_round(4 * B * (4 * nT + 4096)) +
         static_round(4 * 4 * B) + static_round(B * GG) + static_round(8 * B * kAccLanes) + static_round(4 * B) +
         static_round(4 * B * S) + static_round(4 * B * GG) + static_round(2 * B * GG) + static_round(sizeof(FoldEscape) * kFoldEscapes) +
         static_round(4) + static_round(4 * B * S * 8) +
         5 * static_round(8 * B) + 3 * static_round(4 * B) + 2 * static_round(4 * B);
}
static_assert(static_bytes(kStaticMaxVtx, kStaticMaxTri) <= kStaticArenaBytes,
              "the static scratch must hold the largest accepted mesh");

struct StaticLayout {
  float4 *vpos, *vnrm, *xf;
  int4* tri;
  float* rot;
  int *ori, *bin_off, *bin_cur, *bins, *bbox, *flags, *foldcnt, *foldmeta, *o_nbed, *o_flags;
  unsigned *minkey, *trange;
  uint8_t* bedf;
  long long *acc, *o_vo, *o_vss, *o_vtc, *o_ent, *o_col;
  unsigned* foldp;
  short* foldtc;
  FoldEscape* foldx;
  int* foldxn;
  float *o_vof, *o_vssf, *o_vtcf;
  long long bins_total;   // entries of the bins region
};

// Same order and sizes as static_bytes().
StaticLayout static_layout(unsigned char* base, int nV, int nT)
{
  const size_t B = kStaticBatch, GG = (size_t)kStaticGrid * kStaticGrid, S = kStaticGrid;
  size_t off = 0;
  auto take = [&](size_t bytes) { unsigned char* q = base + off; off += static_round(bytes); return (void*)q; };
  StaticLayout L;
  L.vpos = (float4*)take(16 * (size_t)nV);
  L.vnrm = (float4*)take(16 * (size_t)nV);
  L.tri = (int4*)take(16 * (size_t)nT);
  L.rot = (float*)take(4 * 9 * B);
  L.ori = (int*)take(4 * B);
  L.xf = (float4*)take(16 * B * nV);
  L.minkey = (unsigned*)take(4 * 4 * B);
  L.trange = (unsigned*)take(4 * B * nT);
  L.bin_off = (int*)take(4 * B * (S + 1));
  L.bin_cur = (int*)take(4 * B * S);
  L.bins_total = (long long)B * (4 * (long long)nT + 4096);
  L.bins = (int*)take(4 * (size_t)L.bins_total);
  L.bbox = (int*)take(4 * 4 * B);
  L.bedf = (uint8_t*)take(B * GG);
  L.acc = (long long*)take(8 * B * kAccLanes);
  L.flags = (int*)take(4 * B);
  L.foldcnt = (int*)take(4 * B * S);
  L.foldp = (unsigned*)take(4 * B * GG);
  L.foldtc = (short*)take(2 * B * GG);
  L.foldx = (FoldEscape*)take(sizeof(FoldEscape) * kFoldEscapes);
  L.foldxn = (int*)take(4);
  L.foldmeta = (int*)take(4 * B * S * 8);
  L.o_vo = (long long*)take(8 * B); L.o_vss = (long long*)take(8 * B); L.o_vtc = (long long*)take(8 * B);
  L.o_ent = (long long*)take(8 * B); L.o_col = (long long*)take(8 * B);
  L.o_vof = (float*)take(4 * B); L.o_vssf = (float*)take(4 * B); L.o_vtcf = (float*)take(4 * B);
  L.o_nbed = (int*)take(4 * B); L.o_flags = (int*)take(4 * B);
  return L;
}

// Host staging, file-scope so that a call allocates nothing on the host either.
float4 g_static_hpos[kStaticMaxVtx], g_static_hnrm[kStaticMaxVtx];
int4 g_static_htri[kStaticMaxTri];
float g_static_hrot[kStaticBatch * 9];
int g_static_hori[kStaticBatch] = {0, 1, 2, 3};
int g_static_hflags[kStaticBatch], g_static_hnbed[kStaticBatch];
float g_static_hvof[kStaticBatch], g_static_hvssf[kStaticBatch], g_static_hvtcf[kStaticBatch];
float g_static_bedfold[kStaticGrid * kStaticGrid + 1];
void* g_static_addr[kStaticMaxDevices];
static_assert(kStaticBatch == 4, "g_static_hori lists the batch slots");

// Device address of g_static_arena on the current device, looked up once per
// device (with that device current).
int static_arena(void** out)
{
  int dev = 0;
  TOMO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticMaxDevices) return set_error(TOMO_ERR_CAPACITY, "device ordinal beyond the static table");
  if (g_static_addr[dev] == nullptr) {
    void* a = nullptr;
    TOMO_CUDA(cudaGetSymbolAddress(&a, g_static_arena));
    g_static_addr[dev] = a;
  }
  *out = g_static_addr[dev];
  return 0;
}

void static_bind(EngineParams& p, const StaticLayout& L, int nb, int slot, int bin_cap)
{
  p.vpos = L.vpos; p.vnrm = L.vnrm; p.tri = L.tri; p.rot = L.rot;
  p.ori = L.ori + slot; p.Bo = nb;
  p.xf = L.xf; p.minkey = L.minkey; p.trange = L.trange;
  p.bin_off = L.bin_off; p.bin_cur = L.bin_cur; p.bins = L.bins; p.bin_cap = bin_cap;
  p.acc = L.acc; p.flags = L.flags; p.bbox = L.bbox; p.bedf = L.bedf;
  p.foldcnt = L.foldcnt; p.foldp = L.foldp; p.foldmeta = L.foldmeta;
  p.foldtc = p.explicit_ss ? nullptr : L.foldtc;
  p.foldx = L.foldx; p.foldxn = L.foldxn;
  p.out_vo = L.o_vo; p.out_vss = L.o_vss; p.out_vtc = L.o_vtc; p.out_vof = L.o_vof; p.out_vssf = L.o_vssf;
  p.out_vtcf = L.o_vtcf; p.out_nbed = L.o_nbed; p.out_flags = L.o_flags; p.out_entries = L.o_ent;
  p.out_columns = L.o_col;
  p.dump_slot = -1; p.dump_cols = nullptr; p.dump_keys = nullptr; p.dump_types = nullptr;
}

// One batch slot re-run in strip configuration c (Engine::run_subset for a
// single orientation); returns the slot's new status flags or an error.
int static_rerun(Engine& X, const StaticLayout& L, int slot, int c, cudaStream_t st)
{
  X.choose_strips(c);
  const int mode = X.cfg[c].mode;
  EngineParams p = X.base_params(mode);
  p.variant = c;
  const int normal_cap = 4 * X.P.n_tri + 4096;
  static_bind(p, L, 1, slot, mode != 1 ? normal_cap : INT_MAX);
  TOMO_CUDA(cudaMemsetAsync(L.o_nbed + slot, 0, sizeof(int), st));
  if (mode != 1) {
    TOMO_CUDA(launch_batch(p, st, X.cfg[c].smem, nullptr));
  } else {
    TOMO_CUDA(launch_bin_count(p, st, nullptr));
    int total = 0;
    TOMO_CUDA(cudaMemcpyAsync(&total, L.bin_off + X.S, sizeof(int), cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaStreamSynchronize(st));
    if ((long long)total > L.bins_total)
      return set_error(TOMO_ERR_CAPACITY, "tomoSweepStatic: safe-mode strip bins exceed the static scratch");
    p.bin_cap = std::max(total, 1);
    TOMO_CUDA(launch_after_count(p, st, X.cfg[c].smem, nullptr));
  }
  TOMO_CUDA(launch_fold(p, st, nullptr));
  int fl = 0;
  TOMO_CUDA(cudaMemcpyAsync(&fl, L.o_flags + slot, sizeof(int), cudaMemcpyDeviceToHost, st));
  TOMO_CUDA(cudaStreamSynchronize(st));
  return fl;
}

// Synchronizes the call's stream on every return once device work has been
// issued, so that no kernel of a failed call is still queued on the shared
// scratch when the library's lock is released.
struct StreamDrain {
  cudaStream_t st;
  bool armed = false;
  ~StreamDrain()
  {
    if (armed) cudaStreamSynchronize(st);
  }
};

}  // namespace
}  // namespace tomo

extern "C" int tomoSweepStatic(const float* f32info, const int* i32info, const float* YPR, const int* tri,
                               const float* vtx, const float* vtx_nrm, float* Mo, float* Mss, float* Vtc,
                               void* stream)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  if (f32info == nullptr || i32info == nullptr) return set_error(TOMO_ERR_ARG, "info arrays are null");
  const Params P = read_params(f32info, i32info);
  if (P.n_tri < 0 || P.n_vtx < 0 || P.n_ypr < 0) return set_error(TOMO_ERR_ARG, "negative size in Int32Info");
  if (P.n_ypr > 0 && (YPR == nullptr || Mo == nullptr || Mss == nullptr || Vtc == nullptr))
    return set_error(TOMO_ERR_ARG, "YPR or an output array is null");
  if (P.n_tri > 0 && (tri == nullptr || vtx == nullptr || vtx_nrm == nullptr))
    return set_error(TOMO_ERR_ARG, "mesh array is null");
  if (P.n_tri > kStaticMaxTri)
    return set_error(TOMO_ERR_CAPACITY, "tomoSweepStatic: " + std::to_string(P.n_tri) +
                                            " triangles exceed the static limit of " + std::to_string(kStaticMaxTri));
  if (P.n_vtx > kStaticMaxVtx)
    return set_error(TOMO_ERR_CAPACITY, "tomoSweepStatic: " + std::to_string(P.n_vtx) +
                                            " vertices exceed the static limit of " + std::to_string(kStaticMaxVtx));
  for (int t = 0; t < P.n_tri * 3; t++)
    if (tri[t] < 0 || tri[t] >= P.n_vtx) return set_error(TOMO_ERR_ARG, "triangle index out of range");
  for (int k = 0; k < P.n_vtx * 3; k++)
    if (!std::isfinite(vtx[k]) || !std::isfinite(vtx_nrm[k])) return set_error(TOMO_ERR_ARG, "non-finite vertex or normal");
  for (int k = 0; k < P.n_ypr * 3; k++)
    if (!std::isfinite(YPR[k])) return set_error(TOMO_ERR_ARG, "non-finite orientation");
  if (!std::isfinite(P.dVoxel) || !std::isfinite(P.bed_outer) || !std::isfinite(P.theta_c) || P.bed_outer < 0.f ||
      P.bed_outer > 1000.f)
    return set_error(TOMO_ERR_ARG, "bad printer parameters");

  Workspace XW;   // no streams, no buffers: strip planning and kernel parameters only
  Engine X(XW);
  X.P = P;
  X.nYPR = P.n_ypr;
  float mn[3] = {1e5f, 1e5f, 1e5f}, mx[3] = {-1e5f, -1e5f, -1e5f};
  for (int v = 0; v < P.n_vtx; v++)
    for (int k = 0; k < 3; k++) {
      const float d = vtx[v * 3 + k];
      mn[k] = (mn[k] <= d) ? mn[k] : d;
      mx[k] = (mx[k] >= d) ? mx[k] : d;
    }
  X.cx = (float)((double)(mn[0] + mx[0]) * 0.5);
  X.cy = (float)((double)(mn[1] + mx[1]) * 0.5);
  X.cz = (float)((double)(mn[2] + mx[2]) * 0.5);
  X.G = X.choose_grid(vtx, P.n_vtx);
  if (X.G > kStaticGrid)
    return set_error(TOMO_ERR_CAPACITY, "tomoSweepStatic: the mesh footprint needs a slot grid of " +
                                            std::to_string(X.G) + " columns, above the static limit of 256");

  // what Calculate adds per bed pixel, folded (Engine::finalize_host)
  int bedfold_n = 0;
  g_static_bedfold[0] = 0.f;
  auto finish = [&](int id, float vof, float vssf, float vtcf, int nbed) {
    while (bedfold_n < nbed) { g_static_bedfold[bedfold_n + 1] = g_static_bedfold[bedfold_n] + (float)1 * P.bed_thickness; bedfold_n++; }
    float vm[22] = {0};
    vm[8] = vof; vm[4] = vssf; vm[2] = vtcf; vm[11] = g_static_bedfold[nbed];
    vol_to_mass(P, vm);
    Mo[id] = vm[16]; Mss[id] = vm[13]; Vtc[id] = vm[2];
  };
  for (int& r : g_static_reruns) r = 0;
  if (P.n_ypr == 0) return 0;
  if (P.n_tri == 0) {
    for (int i = 0; i < P.n_ypr; i++) finish(i, 0.f, 0.f, 0.f, 0);
    return first_optimal(P.n_ypr, Mss);
  }

  cudaStream_t st = (cudaStream_t)stream;
  StreamDrain drain{st};   // declared after the lock: runs before it is released
  void* base = nullptr;
  TOMO_TRY(static_arena(&base));
  const StaticLayout L = static_layout((unsigned char*)base, P.n_vtx, P.n_tri);
  int dev = 0, optin = 0;
  TOMO_CUDA(cudaGetDevice(&dev));
  TOMO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  X.smem_optin = (size_t)optin;
  X.plan_strips();
  TOMO_TRY(X.configure());

  for (int v = 0; v < P.n_vtx; v++) {
    g_static_hpos[v] = make_float4(vtx[v * 3 + 0], vtx[v * 3 + 1], vtx[v * 3 + 2], 0.f);
    g_static_hnrm[v] = make_float4(vtx_nrm[v * 3 + 0], vtx_nrm[v * 3 + 1], vtx_nrm[v * 3 + 2], 0.f);
  }
  for (int t = 0; t < P.n_tri; t++) g_static_htri[t] = make_int4(tri[t * 3 + 0], tri[t * 3 + 1], tri[t * 3 + 2], 0);
  drain.armed = true;
  TOMO_CUDA(cudaMemcpyAsync(L.vpos, g_static_hpos, sizeof(float4) * P.n_vtx, cudaMemcpyHostToDevice, st));
  TOMO_CUDA(cudaMemcpyAsync(L.vnrm, g_static_hnrm, sizeof(float4) * P.n_vtx, cudaMemcpyHostToDevice, st));
  TOMO_CUDA(cudaMemcpyAsync(L.tri, g_static_htri, sizeof(int4) * P.n_tri, cudaMemcpyHostToDevice, st));
  TOMO_CUDA(cudaMemcpyAsync(L.ori, g_static_hori, sizeof(g_static_hori), cudaMemcpyHostToDevice, st));

  const int normal_cap = 4 * P.n_tri + 4096;
  for (int first = 0; first < P.n_ypr; first += kStaticBatch) {
    const int nb = std::min(kStaticBatch, P.n_ypr - first);
    for (int o = 0; o < nb; o++)
      rotation(YPR[(first + o) * 3 + 0], YPR[(first + o) * 3 + 1], YPR[(first + o) * 3 + 2], &g_static_hrot[o * 9]);
    TOMO_CUDA(cudaMemcpyAsync(L.rot, g_static_hrot, sizeof(float) * 9 * nb, cudaMemcpyHostToDevice, st));
    // out_nbed is accumulated with atomics; every other buffer the kernels
    // read is written first by the batch itself (k_reset clears the rest)
    TOMO_CUDA(cudaMemsetAsync(L.o_nbed, 0, sizeof(int) * nb, st));
    X.choose_strips(0);
    EngineParams p = X.base_params(0);
    static_bind(p, L, nb, 0, normal_cap);
    TOMO_CUDA(launch_batch(p, st, X.cfg[0].smem, nullptr));
    TOMO_CUDA(launch_fold(p, st, nullptr));
    TOMO_CUDA(cudaMemcpyAsync(g_static_hflags, L.o_flags, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaStreamSynchronize(st));
    // the re-run ladder of Engine::resolve_ids, per flagged slot
    for (int o = 0; o < nb; o++) {
      int fl = g_static_hflags[o];
      if (fl & kFlagGrid) return set_error(TOMO_ERR_CAPACITY, "slot index outside the grid");
      bool safe = (fl & (kFlagStray | kFlagBinCap)) != 0;
      if (!safe && (fl & kFlagOverflow)) {
        fl = static_rerun(X, L, o, 2, st);
        if (fl < 0) return fl;
        g_static_reruns[2]++;
        safe = (fl & (kFlagStray | kFlagBinCap | kFlagOverflow)) != 0;
      }
      if (!safe && (fl & kFlagCap)) {
        fl = static_rerun(X, L, o, 4, st);
        if (fl < 0) return fl;
        g_static_reruns[4]++;
        safe = (fl & kFlagRedo) != 0;
      }
      if (safe) {
        fl = static_rerun(X, L, o, 1, st);
        if (fl < 0) return fl;
        g_static_reruns[1]++;
        if (fl & kFlagSafeOverflow) {
          fl = static_rerun(X, L, o, 3, st);
          if (fl < 0) return fl;
          g_static_reruns[3]++;
        }
      }
      if (fl & kFlagSafeOverflow) return set_error(TOMO_ERR_CAPACITY, "column strip exceeds shared memory");
      if (fl & kFlagGrid) return set_error(TOMO_ERR_CAPACITY, "slot index outside the grid");
      if (fl & kFlagRedo) return set_error(TOMO_ERR_CAPACITY, "orientation unresolved after the re-runs");
      if (fl & kFlagFoldRange)
        return set_error(TOMO_ERR_CAPACITY, "column values past 16 bits overflowed the fold escape table");
    }
    TOMO_CUDA(cudaMemcpyAsync(g_static_hvof, L.o_vof, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaMemcpyAsync(g_static_hvssf, L.o_vssf, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaMemcpyAsync(g_static_hvtcf, L.o_vtcf, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaMemcpyAsync(g_static_hnbed, L.o_nbed, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaStreamSynchronize(st));
    for (int o = 0; o < nb; o++) {
      if (g_static_hnbed[o] < 0 || g_static_hnbed[o] > kStaticGrid * kStaticGrid)
        return set_error(TOMO_ERR_CAPACITY, "bed pixel count outside the slot grid");
      finish(first + o, g_static_hvof[o], g_static_hvssf[o], g_static_hvtcf[o], g_static_hnbed[o]);
    }
  }
  return first_optimal(P.n_ypr, Mss);
}

// ------------------------------------------------ multi-mesh batch
//
// Many meshes with uneven triangle counts, each with its own orientation
// list, swept in one CUDA-graph launch: every mesh's batches (reset, rotate,
// bin, strip, bed on the main stream; the fold on the second stream) are
// captured once into a graph over one shared workspace and replayed with a
// single cudaGraphLaunch.  The strip configuration (orientations per batch,
// shared-memory budget) of each mesh is picked by Engine::autotune, once per
// size class (slot-grid edge rounded up to 32, triangle count rounded up to
// a power of two).  Flagged orientations are re-run per mesh afterwards by
// the same ladder as the single-mesh call, so every mesh's results are
// those of TomoSh_CUDA on that mesh alone.

namespace tomo {
namespace {

struct MultiEngine {
  Workspace W;
  std::vector<Engine*> meshes;
  std::vector<int> order;   // capture order: estimated cost, largest first
  std::map<std::pair<int, int>, Engine::TuneResult> tuned;
  std::vector<Engine::TuneResult> choice;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<const void*> graph_ptrs;   // every buffer address the captured graph uses
  size_t graph_nodes = 0;
  long long graph_kernels = 0;
  int autotune = 1;
  int tune_sample = 512;
  int n_tuned = 0;
  double last_ms = 0.0;        // last run: sweep and re-runs, until every mesh is resolved
  double last_graph_ms = 0.0;  // last run: the sweep alone (graph replay)

  void clear_graph()
  {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr; graph = nullptr; graph_nodes = 0; graph_kernels = 0; graph_ptrs.clear();
  }
  void clear_meshes()
  {
    for (auto* e : meshes) { e->release(); delete e; }
    meshes.clear(); order.clear(); choice.clear();
  }
  void release() { clear_graph(); clear_meshes(); W.release(); tuned.clear(); }

  int prepare(int n, const float* const* f32, const int* const* i32, const float* const* ypr, const int* const* tri,
              const float* const* vtx, const float* const* vnrm)
  {
    clear_graph();
    clear_meshes();
    TOMO_TRY(W.init());
    for (int m = 0; m < n; m++) {
      if (f32 == nullptr || i32 == nullptr || f32[m] == nullptr || i32[m] == nullptr)
        return set_error(TOMO_ERR_ARG, "mesh " + std::to_string(m) + ": info arrays are null");
      Engine* e = new Engine(W);
      e->adaptive = 0;   // captured into a graph: no host waits inside the sweep
      meshes.push_back(e);
      const int rc = e->upload(f32[m], i32[m], ypr ? ypr[m] : nullptr, tri ? tri[m] : nullptr, vtx ? vtx[m] : nullptr,
                               vnrm ? vnrm[m] : nullptr);
      if (rc) {
        const std::string why = g_last_error_str;
        clear_meshes();
        return set_error(rc, "mesh " + std::to_string(m) + ": " + why);
      }
    }
    order.resize(n);
    for (int m = 0; m < n; m++) order[m] = m;
    auto cost = [&](int m) {
      const Engine& e = *meshes[m];
      return (double)e.nYPR * ((double)e.P.n_tri + 0.25 * (double)e.G * (double)e.G);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    choice.assign(n, Engine::TuneResult{128, 0, 0, 0, 0.0});
    n_tuned = 0;
    for (int m = 0; m < n; m++) {
      Engine& e = *meshes[m];
      if (!autotune || e.nYPR == 0 || e.P.n_tri == 0) {
        choice[m] = {e.batch, e.normal_smem, e.force_h, e.start_cfg, 0.0};
        continue;
      }
      int t = 1;
      while (t < e.P.n_tri) t <<= 1;
      const std::pair<int, int> key((e.G + 31) / 32 * 32, t);
      auto it = tuned.find(key);
      if (it == tuned.end()) {
        Engine::TuneResult r;
        TOMO_TRY(e.autotune(tune_sample, &r));
        it = tuned.emplace(key, r).first;
        n_tuned++;
      }
      e.batch = it->second.batch;
      e.normal_smem = it->second.normal_smem;
      e.force_h = it->second.strip_h;
      e.start_cfg = it->second.start_cfg;
      e.plan_strips();
      choice[m] = it->second;
    }
    return 0;
  }

  std::vector<const void*> buffer_addresses() const
  {
    std::vector<const void*> v;
    for (const auto& q : W.prep)
      v.insert(v.end(), {q.xf.ptr, q.minkey.ptr, q.trange.ptr, q.bin_off.ptr, q.bin_cur.ptr, q.bins.ptr, q.bbox.ptr,
                         q.bedf.ptr});
    for (const auto& st : W.set) {
      v.insert(v.end(), {st.acc.ptr, st.flags.ptr, st.foldcnt.ptr, st.foldp.ptr, st.foldtc.ptr, st.foldx.ptr, st.foldxn.ptr,
                         st.foldmeta.ptr});
    }
    for (const Engine* e : meshes) {
      v.insert(v.end(), {e->vpos.ptr, e->vnrm.ptr, e->tri.ptr, e->rot.ptr, e->ori.ptr, e->o_vo.ptr, e->o_vss.ptr,
                         e->o_vtc.ptr, e->o_ent.ptr, e->o_col.ptr, e->o_vof.ptr, e->o_vssf.ptr, e->o_vtcf.ptr,
                         e->o_nbed.ptr, e->o_flags.ptr});
    }
    return v;
  }

  // Every buffer the sweep touches, at its final size, before capture.
  int reserve_all()
  {
    for (auto* e : meshes) {
      if (e->nYPR == 0 || e->P.n_tri == 0) continue;
      e->choose_strips(0);
      TOMO_TRY(e->configure());
      TOMO_TRY(e->reserve_outputs());
      TOMO_TRY(e->reserve_batch(std::min(e->batch, e->nYPR), 4 * e->P.n_tri + 4096, e->nYPR > e->batch ? 2 : 1));
    }
    return 0;
  }

  int capture()
  {
    clear_graph();
    const bool timing = W.log.timing;
    long long before = 0;
    for (long long c : W.log.launches) before += c;
    W.log.timing = false;
    TOMO_CUDA(cudaStreamBeginCapture(W.main, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    for (int m : order)
      if ((rc = meshes[m]->sweep_device()) != 0) break;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(W.main, &g);
    W.log.timing = timing;
    long long after = 0;
    for (long long c : W.log.launches) after += c;
    graph_kernels = after - before;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return set_error(TOMO_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    graph = g;
    TOMO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    TOMO_CUDA(cudaGraphGetNodes(graph, nullptr, &graph_nodes));
    return 0;
  }

  int run(int use_graph, float* device_ms)
  {
    if (meshes.empty()) return 0;
    TOMO_TRY(reserve_all());
    // a buffer reallocated since capture (re-runs may grow the bin list)
    // leaves the graph pointing at freed memory: capture it again
    if (exec && graph_ptrs != buffer_addresses()) clear_graph();
    cudaEvent_t a = nullptr, b = nullptr;
    TOMO_CUDA(cudaEventCreate(&a));
    TOMO_CUDA(cudaEventCreate(&b));
    int rc = 0;
    if (use_graph && !exec) {
      rc = capture();
      graph_ptrs = buffer_addresses();
    }
    if (rc == 0 && cudaEventRecord(a, W.main) != cudaSuccess) rc = set_error(TOMO_ERR_CUDA, "event record");
    if (rc == 0) {
      if (use_graph) {
        const cudaError_t e = cudaGraphLaunch(exec, W.main);
        if (e != cudaSuccess) rc = set_error(TOMO_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
      } else {
        for (int m : order)
          if ((rc = meshes[m]->sweep_device()) != 0) break;
      }
    }
    // the sweep alone (graph) ends at g; the re-runs of flagged orientations
    // follow per mesh on the same stream, and b marks every mesh resolved
    cudaEvent_t g = nullptr;
    if (rc == 0 && (cudaEventCreate(&g) != cudaSuccess || cudaEventRecord(g, W.main) != cudaSuccess))
      rc = set_error(TOMO_ERR_CUDA, "event record");
    for (auto* e : meshes)
      if (rc == 0) rc = e->resolve();
    float ms = 0.f, gms = 0.f;
    if (rc == 0) {
      if (cudaEventRecord(b, W.main) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess ||
          cudaEventElapsedTime(&ms, a, b) != cudaSuccess || cudaEventElapsedTime(&gms, a, g) != cudaSuccess)
        rc = set_error(TOMO_ERR_CUDA, "batch timing");
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (g) cudaEventDestroy(g);
    if (rc) return rc;
    last_ms = ms;
    last_graph_ms = gms;
    if (device_ms) *device_ms = ms;
    for (auto* e : meshes) e->finalize_host();
    return 0;
  }
};

MultiEngine* g_multi = nullptr;

MultiEngine& multi()
{
  if (!g_multi) g_multi = new MultiEngine();
  return *g_multi;
}

}  // namespace
}  // namespace tomo

extern "C" {

int tomoBatchPrepare(int n_mesh, const float* const* f32info, const int* const* i32info, const float* const* YPR,
                     const int* const* tri, const float* const* vtx, const float* const* vtx_nrm)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  if (n_mesh < 0) return set_error(TOMO_ERR_ARG, "negative mesh count");
  return multi().prepare(n_mesh, f32info, i32info, YPR, tri, vtx, vtx_nrm);
}

int tomoBatchRun(int use_graph, float* device_ms)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  if (!g_multi) return set_error(TOMO_ERR_ARG, "tomoBatchPrepare was not called");
  return g_multi->run(use_graph, device_ms);
}

int tomoBatchResults(int mesh, float* Mo, float* Mss, float* Vtc, long long* vo64, long long* vss64, long long* vtc64)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_multi || mesh < 0 || mesh >= (int)g_multi->meshes.size()) return set_error(TOMO_ERR_ARG, "bad mesh index");
  const Engine& E = *g_multi->meshes[mesh];
  const size_t n = (size_t)E.nYPR;
  if (E.Mss.size() < n) return set_error(TOMO_ERR_ARG, "tomoBatchRun was not called");
  if (Mo) std::memcpy(Mo, E.Mo.data(), sizeof(float) * n);
  if (Mss) std::memcpy(Mss, E.Mss.data(), sizeof(float) * n);
  if (Vtc) std::memcpy(Vtc, E.Vtc.data(), sizeof(float) * n);
  if (vo64 && E.vo64.size() >= n) std::memcpy(vo64, E.vo64.data(), sizeof(long long) * n);
  if (vss64 && E.vss64.size() >= n) std::memcpy(vss64, E.vss64.data(), sizeof(long long) * n);
  if (vtc64 && E.vtc64.size() >= n) std::memcpy(vtc64, E.vtc64.data(), sizeof(long long) * n);
  return first_optimal((int)n, E.Mss.data());
}

int tomoBatchStats(long long* out, int n)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_multi || out == nullptr) return TOMO_ERR_ARG;
  const MultiEngine& M = *g_multi;
  long long orient = 0, redo = 0;
  for (auto* e : M.meshes) { orient += e->nYPR; redo += e->n_redo[1] + e->n_redo[2] + e->n_redo[3] + e->n_redo[4]; }
  const long long v[9] = {(long long)M.meshes.size(), orient, (long long)M.graph_nodes, M.graph_kernels,
                          (long long)M.n_tuned, (long long)M.tuned.size(), redo, (long long)(M.last_ms * 1000.0),
                          (long long)(M.last_graph_ms * 1000.0)};
  for (int k = 0; k < n && k < 9; k++) out[k] = v[k];
  return 0;
}

int tomoBatchConfig(int mesh, int* out4)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_multi || mesh < 0 || mesh >= (int)g_multi->meshes.size() || out4 == nullptr)
    return set_error(TOMO_ERR_ARG, "bad mesh index");
  const Engine& E = *g_multi->meshes[mesh];
  out4[0] = E.batch;
  out4[1] = E.normal_smem;
  out4[2] = E.cfg[0].H;
  out4[3] = E.G;
  return 0;
}

int TomoSh_CUDA_Batch(int n_mesh, const float* const* f32info, const int* const* i32info, const float* const* YPR,
                      const int* const* tri, const float* const* vtx, const float* const* vtx_nrm, int* optIDs)
{
  int rc = tomoBatchPrepare(n_mesh, f32info, i32info, YPR, tri, vtx, vtx_nrm);
  if (rc) return rc;
  rc = tomoBatchRun(1, nullptr);
  if (rc) return rc;
  for (int m = 0; m < n_mesh; m++) {
    const int o = tomoBatchResults(m, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (o < 0) return o;
    if (optIDs) optIDs[m] = o;
  }
  return 0;
}

// The TomoSh_CUDA tail for mesh `mesh` of the last batch run: its optID's
// render pixels, vm_info and mat4x4 go to the reference getters (getMss /
// getMo / getVtc return this mesh's arrays), as if TomoSh_CUDA had just run
// on it alone.  Returns the optID.
int tomoBatchExport(int mesh)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  if (!g_multi || mesh < 0 || mesh >= (int)g_multi->meshes.size()) return set_error(TOMO_ERR_ARG, "bad mesh index");
  Engine& E = *g_multi->meshes[mesh];
  const int n = E.nYPR;
  if ((int)E.Mss.size() < n) return set_error(TOMO_ERR_ARG, "tomoBatchRun was not called");
  g_Mss.assign(E.Mss.begin(), E.Mss.begin() + n);
  g_Mo.assign(E.Mo.begin(), E.Mo.begin() + n);
  g_Vtc.assign(E.Vtc.begin(), E.Vtc.begin() + n);
  g_Vo64 = E.vo64; g_Vss64 = E.vss64; g_Vtc64 = E.vtc64;
  const int opt = first_optimal(n, g_Mss.data());
  std::memset(g_volmass, 0, sizeof(g_volmass));
  for (int k = 0; k < 11; k++) { g_pix[k].clear(); g_npix[k] = 0; }
  if (n > 0) {
    if (E.P.n_tri > 0) {
      const int rc = export_best(E, opt, g_pix, g_npix, g_volmass);
      if (rc) return rc;
    } else {
      g_volmass[2] = E.vtcf[opt];
    }
    g_volmass[8] = E.vof[opt]; g_volmass[4] = E.vssf[opt];
    vol_to_mass(E.P, g_volmass);
    host_mat4x4(E, E.h_vtx.data(), E.P.n_vtx, opt, g_mat4x4);
  }
  return opt;
}

void tomoBatchRelease(void)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_multi) { g_multi->release(); delete g_multi; g_multi = nullptr; }
}

int tomoBatchSetOption(int key, int value)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  switch (key) {
    case 1: multi().autotune = value ? 1 : 0; return 0;
    case 2: if (value < 1) return TOMO_ERR_ARG; multi().tune_sample = value; return 0;
    default: return TOMO_ERR_ARG;
  }
}

}  // extern "C"

// ------------------------------------------------ learned-proposal search
//
// The orientation grid is YPR[n_pitch][n_yaw] (yaw fastest), cut into cells
// of cell x cell grid points.  The exact kernels evaluate the coarse points
// (both grid indices multiples of `cell`); the MLP of tomo_mlp.cu is trained
// on their exact Vss (standardised) from [sin y, cos y, sin p, cos p],
// predicts Vss on every grid point, and the cells are ranked by their
// smallest prediction.  The top_k cells are evaluated exactly.  The largest
// prediction error seen on those out-of-sample points, err, then decides
// which other cells could still hold something better than the best exact
// Vss found: every cell whose smallest prediction is within err of it is
// evaluated too, round after round.  If that would take more than
// max_expand cells, or the mean relative error on the refined points
// exceeds `gate`, the search falls back to the exhaustive sweep.  With the
// bed off, Mss is a non-decreasing function of Vss (VolToMass), so ranking
// by Vss ranks by Mss; with a bed the search always falls back.  The answer
// is _find1stOptimal over the evaluated orientations in grid order.

namespace tomo {
namespace {

Mlp* g_mlp = nullptr;

Mlp& mlp()
{
  if (!g_mlp) g_mlp = new Mlp();
  return *g_mlp;
}

double seconds_since(std::chrono::steady_clock::time_point t0)
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Exact evaluation of `ids` on the device (configuration 0 plus the re-run ladder).
int eval_ids(Engine& E, const std::vector<int>& ids, DevBuf<int>& dids)
{
  if (ids.empty()) return 0;
  TOMO_TRY(E.ensure_rot(ids));
  TOMO_CUDA(dids.reserve(ids.size()));
  TOMO_CUDA(cudaMemcpyAsync(dids.ptr, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice, E.main));
  TOMO_TRY(E.sweep_device(dids.ptr, (int)ids.size()));
  TOMO_TRY(E.resolve(&ids));
  return 0;
}

}  // namespace
}  // namespace tomo

extern "C" {

int tomoMlpInit(int seed)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  Engine& E = engine();
  TOMO_TRY(E.init());
  TOMO_CUDA(mlp().init((unsigned)seed, E.main));
  return mlp().param_count();
}

int tomoMlpParams(float* get, const float* set)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_mlp) return set_error(TOMO_ERR_ARG, "tomoMlpInit was not called");
  Engine& E = engine();
  if (set) TOMO_CUDA(mlp().set_params(set, E.main));
  if (get) TOMO_CUDA(mlp().get_params(get, E.main));
  return mlp().param_count();
}

int tomoMlpGrad(const float* x, const float* y, int n, float* grad, float* loss)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_mlp) return set_error(TOMO_ERR_ARG, "tomoMlpInit was not called");
  if (n <= 0 || x == nullptr || y == nullptr) return set_error(TOMO_ERR_ARG, "empty training data");
  Engine& E = engine();
  TOMO_CUDA(mlp().set_data(x, y, n, E.main));
  TOMO_CUDA(mlp().grad(E.main));
  TOMO_CUDA(mlp().read_grad(grad, loss, E.main));
  return 0;
}

int tomoMlpAdam(float lr)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_mlp) return set_error(TOMO_ERR_ARG, "tomoMlpInit was not called");
  Engine& E = engine();
  TOMO_CUDA(mlp().adam(lr, E.main));
  TOMO_CUDA(cudaStreamSynchronize(E.main));
  return 0;
}

int tomoMlpFit(const float* x, const float* y, int n, int steps, float lr, float* loss)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_mlp) return set_error(TOMO_ERR_ARG, "tomoMlpInit was not called");
  if (n <= 0 || x == nullptr || y == nullptr || steps < 0) return set_error(TOMO_ERR_ARG, "bad training arguments");
  Engine& E = engine();
  TOMO_CUDA(mlp().set_data(x, y, n, E.main));
  TOMO_CUDA(mlp().fit(steps, lr, E.main, loss));
  return 0;
}

int tomoMlpPredict(const float* x, int n, float* out)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_mlp) return set_error(TOMO_ERR_ARG, "tomoMlpInit was not called");
  if (n <= 0 || x == nullptr || out == nullptr) return set_error(TOMO_ERR_ARG, "bad prediction arguments");
  Engine& E = engine();
  DevBuf<float> dx, dy;
  TOMO_CUDA(dx.reserve((size_t)n * kMlpIn));
  TOMO_CUDA(dy.reserve((size_t)n));
  TOMO_CUDA(cudaMemcpyAsync(dx.ptr, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, E.main));
  TOMO_CUDA(mlp().predict_device(dx.ptr, n, dy.ptr, E.main));
  TOMO_CUDA(cudaMemcpyAsync(out, dy.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, E.main));
  TOMO_CUDA(cudaStreamSynchronize(E.main));
  dx.release();
  dy.release();
  return 0;
}

int tomoSurrogateSearch(const float* f32info, const int* i32info, const float* YPR, const int* tri, const float* vtx,
                        const float* vtx_nrm, int n_yaw, int n_pitch, const int* iparams, const float* fparams,
                        float* Mss_out, float* pred_out, double* stats)
{
  std::lock_guard<std::mutex> lock(g_mutex);
  g_last_error = 0; g_last_error_str.clear();
  const auto t_start = std::chrono::steady_clock::now();
  if (f32info == nullptr || i32info == nullptr || iparams == nullptr || fparams == nullptr)
    return set_error(TOMO_ERR_ARG, "null argument");
  const int stride = iparams[0], cell = iparams[1], top_k = iparams[2], steps = iparams[3], seed = iparams[4];
  const float lr = fparams[0], gate = fparams[1], margin = fparams[2], holdout = fparams[3], log_scale = fparams[4];
  if (n_yaw <= 0 || n_pitch <= 0 || (long long)n_yaw * n_pitch != i32info[6])
    return set_error(TOMO_ERR_ARG, "n_yaw * n_pitch must equal nYPR");
  if (stride < 1 || cell < 1 || top_k < 1 || steps < 0 || iparams[5] < 0 || !(margin >= 0.f) || !(holdout >= 0.f) ||
      holdout >= 0.9f)
    return set_error(TOMO_ERR_ARG, "bad search parameters");
  Engine& E = engine();
  TOMO_TRY(E.init());
  TOMO_TRY(E.upload(f32info, i32info, YPR, tri, vtx, vtx_nrm, true));
  const int n = E.nYPR;
  const int budget = iparams[5] > 0 ? iparams[5] : std::max(1, n / 5);
  double t_exact = 0.0, t_train = 0.0, t_pred = 0.0;
  std::vector<char> done(n, 0), trained(n, 0);
  std::vector<int> evaluated;
  DevBuf<int> dids;
  auto evaluate = [&](const std::vector<int>& ids) -> int {
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = eval_ids(E, ids, dids);
    t_exact += seconds_since(t0);
    if (rc) return rc;
    for (int i : ids) { done[i] = 1; evaluated.push_back(i); }
    return 0;
  };
  const int ncy = (n_yaw + cell - 1) / cell, ncp = (n_pitch + cell - 1) / cell, ncell = ncy * ncp;
  auto cell_of = [&](int id) { return (id % n_yaw) / cell + ((id / n_yaw) / cell) * ncy; };
  std::vector<float> pred(n, 0.f);
  double rel_err = 0.0, max_err = 0.0;
  float train_loss = 0.f;
  int fallback = 0, rounds = 0, cells_refined = 0, n_coarse = 0;

  if (E.P.bed_type != kBedNone || E.P.n_tri == 0) {
    fallback = 1;
  } else {
    // 1. coarse points (both grid indices multiples of `stride`), exact
    std::vector<int> coarse;
    for (int ip = 0; ip < n_pitch; ip += stride)
      for (int iy = 0; iy < n_yaw; iy += stride) coarse.push_back(ip * n_yaw + iy);
    n_coarse = (int)coarse.size();
    TOMO_TRY(evaluate(coarse));
    // bilinear interpolation of the exact coarse Vss onto every grid point
    // (yaw wraps around): the proposal of the search without the network
    auto interpolate = [&](std::vector<float>& out) {
      const int ncyc = (n_yaw + stride - 1) / stride, ncpc = (n_pitch + stride - 1) / stride;
      auto cval = [&](int p, int y) { return (double)E.vss64[(size_t)(p * stride) * n_yaw + (size_t)(y * stride)]; };
      for (int ip = 0; ip < n_pitch; ip++) {
        const double fp = std::min((double)ip / stride, (double)(ncpc - 1));
        const int p0 = (int)std::floor(fp), p1 = std::min(p0 + 1, ncpc - 1);
        const double wp = fp - p0;
        for (int iy = 0; iy < n_yaw; iy++) {
          const double fy = (double)iy / stride;
          const int y0 = (int)std::floor(fy) % ncyc, y1 = (y0 + 1) % ncyc;
          const double wy = fy - std::floor(fy);
          const double r0 = cval(p0, y0) * (1.0 - wy) + cval(p0, y1) * wy;
          const double r1 = cval(p1, y0) * (1.0 - wy) + cval(p1, y1) * wy;
          out[(size_t)ip * n_yaw + iy] = (float)((1.0 - wp) * r0 + wp * r1);
        }
      }
    };
    if (g_proposal == 1) {
      // 2'-3'. the search without the network; the coarse points are exact,
      // so the error is measured on the refined points only
      const auto t0 = std::chrono::steady_clock::now();
      interpolate(pred);
      for (int id : coarse) trained[id] = 1;
      t_pred += seconds_since(t0);
    } else {
      // 2. features of every grid point on the device (the same bits for
      //    training and prediction); a seeded share of the coarse points is
      //    held out of training so the prediction error is also measured away
      //    from the refined cells; train on standardised exact Vss
      const auto t_feat = std::chrono::steady_clock::now();
      DevBuf<float>& dypr = E.srch_ypr;
      DevBuf<float>& dx = E.srch_x;
      DevBuf<float>& dy = E.srch_y;
      TOMO_CUDA(dypr.reserve((size_t)n * 3));
      TOMO_CUDA(dx.reserve((size_t)n * kMlpIn));
      TOMO_CUDA(dy.reserve((size_t)n));
      TOMO_CUDA(cudaMemcpyAsync(dypr.ptr, YPR, sizeof(float) * n * 3, cudaMemcpyHostToDevice, E.main));
      TOMO_CUDA(mlp_features(dypr.ptr, n, dx.ptr, E.main));
      std::vector<float> F((size_t)n * kMlpIn);
      TOMO_CUDA(cudaMemcpyAsync(F.data(), dx.ptr, sizeof(float) * F.size(), cudaMemcpyDeviceToHost, E.main));
      TOMO_CUDA(cudaStreamSynchronize(E.main));
      t_pred += seconds_since(t_feat);
      std::vector<int> train;
      {
        unsigned h = 2166136261u ^ (unsigned)seed;
        for (int id : coarse) {
          h = (h ^ (unsigned)id) * 16777619u;   // FNV-1a step: a fixed pseudo-random split
          const float u = (float)((h >> 8) & 0xFFFF) / 65536.f;
          if (u >= holdout) { train.push_back(id); trained[id] = 1; }
        }
        if (train.empty()) { train = coarse; for (int id : coarse) trained[id] = 1; }
      }
      // target: Vss, or with log_scale > 0 log1p((Vss - min) / s), s = log_scale x
      // (median - min) of the training Vss, which spends the network's accuracy
      // near the minimum; then standardised
      std::vector<double> tv;
      for (int id : train) tv.push_back((double)E.vss64[id]);
      std::vector<double> sorted_tv = tv;
      std::sort(sorted_tv.begin(), sorted_tv.end());
      const double vmin = sorted_tv.front();
      const double tscale = log_scale > 0.f ? std::max(1.0, (double)log_scale * (sorted_tv[sorted_tv.size() / 2] - vmin)) : 0.0;
      auto fwd = [&](double v) { return tscale > 0.0 ? std::log1p((v - vmin) / tscale) : v; };
      auto inv = [&](double y) { return tscale > 0.0 ? vmin + tscale * std::expm1(y) : y; };
      double mean = 0.0, sq = 0.0;
      for (double v : tv) mean += fwd(v);
      mean /= (double)tv.size();
      for (double v : tv) sq += (fwd(v) - mean) * (fwd(v) - mean);
      const double sd = tv.size() > 1 && sq > 0.0 ? std::sqrt(sq / (double)tv.size()) : 1.0;
      std::vector<float> X(train.size() * kMlpIn), Y(train.size());
      for (size_t k = 0; k < train.size(); k++) {
        std::memcpy(&X[k * kMlpIn], &F[(size_t)train[k] * kMlpIn], sizeof(float) * kMlpIn);
        Y[k] = (float)((fwd(tv[k]) - mean) / sd);
      }
      {
        const auto t0 = std::chrono::steady_clock::now();
        TOMO_CUDA(mlp().init((unsigned)seed, E.main));
        TOMO_CUDA(mlp().set_data(X.data(), Y.data(), (int)train.size(), E.main));
        TOMO_CUDA(mlp().fit(steps, lr, E.main, &train_loss));
        t_train += seconds_since(t0);
      }
      // 3. predict every grid point
      {
        const auto t0 = std::chrono::steady_clock::now();
        TOMO_CUDA(mlp().predict_device(dx.ptr, n, dy.ptr, E.main));
        TOMO_CUDA(cudaMemcpyAsync(pred.data(), dy.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, E.main));
        TOMO_CUDA(cudaStreamSynchronize(E.main));
        for (int id = 0; id < n; id++) pred[id] = (float)inv(pred[id] * sd + mean);
        if (g_proposal == 2) {   // the network and the interpolation, averaged
          std::vector<float> lin(n);
          interpolate(lin);
          for (int id = 0; id < n; id++) pred[id] = 0.5f * (pred[id] + lin[id]);
        }
        t_pred += seconds_since(t0);
      }
    }
    // 4. cells by smallest prediction; refine the top_k
    std::vector<float> cmin(ncell, INFINITY);
    for (int id = 0; id < n; id++) { const int c = cell_of(id); cmin[c] = std::min(cmin[c], pred[id]); }
    std::vector<int> rank(ncell);
    for (int c = 0; c < ncell; c++) rank[c] = c;
    std::stable_sort(rank.begin(), rank.end(), [&](int a, int b) { return cmin[a] < cmin[b]; });
    std::vector<char> refined(ncell, 0);
    std::vector<int> cell_todo(ncell, 0);
    for (int id = 0; id < n; id++) if (!done[id]) cell_todo[cell_of(id)]++;
    auto refine_cells = [&](const std::vector<int>& cells) -> int {
      std::vector<int> ids;
      for (int c : cells) refined[c] = 1;
      for (int id = 0; id < n; id++)
        if (!done[id] && refined[cell_of(id)]) ids.push_back(id);
      cells_refined += (int)cells.size();
      return evaluate(ids);
    };
    std::vector<int> first(rank.begin(), rank.begin() + std::min(top_k, ncell));
    TOMO_TRY(refine_cells(first));
    // 5. error gate and expansion: every untrained evaluated point (held-out
    //    coarse points and refined points) measures the prediction error
    for (;; rounds++) {
      double sum_abs = 0.0, sum_ref = 0.0;
      max_err = 0.0;
      long long best = LLONG_MAX;
      int m = 0;
      for (int id : evaluated) {
        best = std::min(best, E.vss64[id]);
        if (trained[id]) continue;
        const double e = std::fabs((double)pred[id] - (double)E.vss64[id]);
        max_err = std::max(max_err, e);
        sum_abs += e;
        sum_ref += std::fabs((double)E.vss64[id]);
        m++;
      }
      rel_err = m ? sum_abs / std::max(sum_ref, 1.0) : 0.0;
      if (rel_err > gate) { fallback = 1; break; }
      std::vector<int> more;
      long long extra = 0;
      for (int c : rank)
        if (!refined[c] && (double)cmin[c] - margin * max_err <= (double)best) { more.push_back(c); extra += cell_todo[c]; }
      if (more.empty()) break;
      if ((long long)evaluated.size() + extra > budget) { fallback = 1; break; }
      TOMO_TRY(refine_cells(more));
    }
  }
  if (fallback) {
    // the exhaustive sweep itself, over the whole grid
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<int> all(n);
    for (int id = 0; id < n; id++) all[id] = id;
    TOMO_TRY(E.ensure_rot(all));
    TOMO_TRY(E.sweep_device());
    TOMO_TRY(E.resolve());
    t_exact += seconds_since(t0);
    for (int id = 0; id < n; id++) if (!done[id]) { done[id] = 1; evaluated.push_back(id); }
  }
  E.finalize_host();
  // _find1stOptimal over the evaluated orientations, in grid order
  int opt = 0;
  if (n > 1) {
    float bestm = 1e5f;
    for (int id = 0; id < n; id++)
      if (done[id] && E.Mss[id] < bestm) { bestm = E.Mss[id]; opt = id; }
  }
  if (Mss_out)
    for (int id = 0; id < n; id++) Mss_out[id] = done[id] ? E.Mss[id] : NAN;
  if (pred_out) std::memcpy(pred_out, pred.data(), sizeof(float) * n);
  if (stats) {
    const double v[12] = {(double)evaluated.size(), (double)fallback, rel_err, max_err, (double)train_loss,
                          seconds_since(t_start), t_exact, t_train, t_pred, (double)cells_refined, (double)rounds,
                          (double)n_coarse};
    std::memcpy(stats, v, sizeof(v));
  }
  return opt;
}

}  // extern "C"
