// TEST INFRASTRUCTURE ONLY: a thin driver over the reference INT3 engine.
//
// This translation unit is compiled together with the *unmodified* reference
// CPU sources (cfms_tomo/Tomo_Shell_vc_src/cpu_src/*.cpp, Tomo_types.cpp) into
// oracle/_ref/libtomo_ref.so.  It is the reference itself, driven from C:
// the per-orientation step sequence, the thread fan-out and the argmin follow
// _TomoSh_Function_Call / thread_func / _find1stOptimal
// (cfms_tomo/Tomo_Shell_vc_src/Tomo_Shell2026.cpp:89-248).  Two additions,
// both read-only with respect to the engine's arithmetic:
//
//   * exact int64 per-orientation totals of the per-column Vo/Vss, summed
//     from the paired slot buffer with the same type-bit rule as the
//     reference's own debug accumulator tomoCalcCpuSlotPairSums
//     (cpu_src/STomoSh_INT3.cpp:129-170), because vm_info.Vo/Vss are float32
//     accumulators (cpu_src/STomoVolMassInfo.h:24-31);
//   * an optional square slot grid larger than the engine's hard-wired
//     256x256 (cpu_src/STomoVoxelSpaceInfo.h:10), set through the engine's
//     public SetMem().  The engine does no bounds checks, so meshes whose
//     rotated footprint exceeds 256 columns need it; grid size does not
//     change any arithmetic.
//
// Nothing here is linked into the product library.
#include "pch.h"
#include "cpu_src/STomoSh_INT3.h"

#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using namespace Tomo;

namespace {

// Per-column (Vo, Vss) from a paired slot, type-bit rule of
// tomoCalcCpuSlotPairSums (cpu_src/STomoSh_INT3.cpp:129-170).
void slotSums(const STomoSh_INT3& nv, const SLOT_BUFFER_TYPE* slot, int& vo, int& vss, int& tc)
{
  vo = 0; vss = 0; tc = 0;
  const int S_L = slot[0];
  if (S_L <= 1) return;
  const int S_W = nv.voxel_info.nSlotCapacityWidth;
  int al = 0, be = 0, ssb = 0, ssa = 0, t = 0, nvb = 0, nva = 0;
  for (int p = 0; p < S_L; p++) {
    const int type = slot[(p + 1) * S_W + 0];
    const int z = slot[(p + 1) * S_W + 1];
    if (type & typeAl) {
      al += z;
      if (type & typeTC) t += z;
      if (type & typeNVA) nva += z;
    } else if (type & typeBe) {
      be += z;
      if (type & typeNVB) nvb += z;
    }
    if (type & typeSSB) ssb += z;
    else if (type & typeSSA) ssa += z;
  }
  vo = (al > be) ? (al - be) : 0;
  vss = nv.printer_info.bUseExplicitSS ? (ssb - ssa) : (-al + be + t - nvb + nva);
  tc = t;
}

struct SweepOut {
  float* Mo; float* Mss; float* Vtc; float* VoF; float* VssF;
  long long* Vo64; long long* Vss64; long long* Vtc64;
};

// thread_func (Tomo_Shell2026.cpp:99-117) plus the int64 side channel.
void runOne(STomoSh_INT3* nv, const float* ypr, int id, const SweepOut& o)
{
  S3DPrinterInfo& info = nv->printer_info;
  info.yaw = ypr[id * 3 + 0];
  info.pitch = ypr[id * 3 + 1];
  info.roll = ypr[id * 3 + 2];

  nv->Rotate();
  nv->Pixelize();
  nv->Pairing();
  if (o.Vo64 != nullptr) {
    const int S_W = nv->voxel_info.nSlotCapacityWidth;
    const int S_H = nv->voxel_info.nSlotCapacityHeight;
    long long vo = 0, vss = 0, tc = 0;
    for (size_t i = 0; i < nv->voxel_info.dirtySlots.size(); i++) {
      const SLOT_BUFFER_TYPE* slot = nv->voxel_info.SlotBuf_108f + nv->voxel_info.dirtySlots[i] * S_W * S_H;
      int a, b, c;
      slotSums(*nv, slot, a, b, c);
      vo += a; vss += b; tc += c;
    }
    o.Vo64[id] = vo;
    o.Vss64[id] = vss;
    if (o.Vtc64 != nullptr) o.Vtc64[id] = tc;
  }
  if (o.VoF != nullptr) o.VoF[id] = nv->vm_info.Vo;
  if (o.VssF != nullptr) o.VssF[id] = nv->vm_info.Vss;
  nv->GenerateBed();
  nv->Calculate();

  o.Mo[id] = nv->vm_info.Mo;
  o.Mss[id] = nv->vm_info.Mss;
  o.Vtc[id] = nv->vm_info.Vtc;
}

// _find1stOptimal (Tomo_Shell2026.cpp:89-97).
int firstOptimal(int n, const float* mss)
{
  if (n <= 1) return 0;
  int idx = 0;
  float best = 1e5f;
  for (int i = 0; i < n; i++) {
    if (mss[i] < best) { best = mss[i]; idx = i; }
  }
  return idx;
}

void prepare(STomoSh_INT3* pNV, int n, const S3DPrinterInfo& info, int grid)
{
  for (int i = 0; i < n; i++) {
    pNV[i].printer_info = info;
    if (grid > 0 && grid != pNV[i].voxel_info.x_dim) pNV[i].voxel_info.SetMem(grid, grid, pNV[i].voxel_info.z_dim);
  }
}

}  // namespace

extern "C" {

// Full orientation sweep through the reference INT3 engine.  Orchestration
// follows _TomoSh_Function_Call (Tomo_Shell2026.cpp:194-215): blocks of
// n_threads std::threads, one orientation each, joined per block.  Returns
// the reference optID.  Vo64/Vss64/Vtc64/VoF/VssF may be null.
int ref_int3_sweep(const float* f32info, const int* i32info, const float* ypr,
                   const int* tri, const float* vtx, const float* vnrm, const float* tnrm,
                   const int* htri, const float* hvtx, const float* htnrm,
                   int grid, int n_threads,
                   float* Mo, float* Mss, float* Vtc, float* VoF, float* VssF,
                   long long* Vo64, long long* Vss64, long long* Vtc64)
{
  S3DPrinterInfo info(const_cast<float*>(f32info), const_cast<int*>(i32info), const_cast<int*>(tri),
                      const_cast<float*>(vtx), const_cast<float*>(vnrm), const_cast<float*>(tnrm),
                      const_cast<int*>(htri), const_cast<float*>(hvtx), const_cast<float*>(htnrm), 0, 0, 0);
  const int nYPR = static_cast<int>(info.nYPR);
  int nThread = n_threads < 1 ? 1 : n_threads;
  if (nYPR < nThread) nThread = nYPR;
  if (nThread < 1) nThread = 1;
  const int nBlock = nYPR / nThread;
  const int nRest = nYPR % nThread;

  std::vector<STomoSh_INT3> pool(nThread);
  prepare(pool.data(), nThread, info, grid);
  SweepOut o{Mo, Mss, Vtc, VoF, VssF, Vo64, Vss64, Vtc64};

  int id = 0;
  for (int b = 0; b < nBlock; b++) {
    std::vector<std::thread> th;
    for (int t = 0; t < nThread; t++) th.emplace_back(runOne, &pool[t], ypr, id++, o);
    for (auto& x : th) x.join();
  }
  {
    std::vector<std::thread> th;
    for (int t = 0; t < nRest; t++) th.emplace_back(runOne, &pool[t], ypr, id++, o);
    for (auto& x : th) x.join();
  }
  return firstOptimal(nYPR, Mss);
}

// One orientation through the reference engine with per-column dumps.
//   n_vox[g*g]           slot count right after Pixelize
//   vox_zn[g*g*64*2]     (z, nz) per slot in insertion order after Pixelize
//   n_fin[g*g]           slot count after Pairing + GenerateBed (sentinels, bed)
//   fin_tzn[g*g*64*3]    (type, z, nz) per slot after Pairing + GenerateBed
//   col_vo, col_vss      per-column values (tomoCalcCpuSlotPairSums rule)
//   volmass22            vm_info.dData after Calculate
//   mat16                mat4x4.Data after Rotate
// Any output pointer may be null.  Returns 0.
int ref_int3_columns(const float* f32info, const int* i32info, const float* ypr,
                     const int* tri, const float* vtx, const float* vnrm, const float* tnrm,
                     const int* htri, const float* hvtx, const float* htnrm,
                     int ypr_index, int grid,
                     int* n_vox, short* vox_zn, int* n_fin, short* fin_tzn,
                     int* col_vo, int* col_vss, float* volmass22, float* mat16)
{
  S3DPrinterInfo info(const_cast<float*>(f32info), const_cast<int*>(i32info), const_cast<int*>(tri),
                      const_cast<float*>(vtx), const_cast<float*>(vnrm), const_cast<float*>(tnrm),
                      const_cast<int*>(htri), const_cast<float*>(hvtx), const_cast<float*>(htnrm), 0, 0, 0);
  STomoSh_INT3* nv = new STomoSh_INT3[1];
  prepare(nv, 1, info, grid);
  S3DPrinterInfo& pi = nv->printer_info;
  pi.yaw = ypr[ypr_index * 3 + 0];
  pi.pitch = ypr[ypr_index * 3 + 1];
  pi.roll = ypr[ypr_index * 3 + 2];

  const int X_D = nv->voxel_info.x_dim;
  const int Y_D = nv->voxel_info.y_dim;
  const int S_W = nv->voxel_info.nSlotCapacityWidth;
  const int S_H = nv->voxel_info.nSlotCapacityHeight;
  const SLOT_BUFFER_TYPE* buf = nv->voxel_info.SlotBuf_108f;

  nv->Rotate();
  nv->Pixelize();
  for (int s = 0; s < X_D * Y_D; s++) {
    const SLOT_BUFFER_TYPE* slot = buf + static_cast<size_t>(s) * S_W * S_H;
    if (n_vox != nullptr) n_vox[s] = slot[0];
    if (vox_zn != nullptr) {
      for (int p = 0; p < S_H; p++) {
        const bool live = p < slot[0];
        vox_zn[(static_cast<size_t>(s) * S_H + p) * 2 + 0] = live ? slot[(p + 1) * S_W + 1] : 0;
        vox_zn[(static_cast<size_t>(s) * S_H + p) * 2 + 1] = live ? slot[(p + 1) * S_W + 2] : 0;
      }
    }
  }
  nv->Pairing();
  for (int s = 0; s < X_D * Y_D; s++) {
    const SLOT_BUFFER_TYPE* slot = buf + static_cast<size_t>(s) * S_W * S_H;
    int a, b, c;
    slotSums(*nv, slot, a, b, c);
    if (col_vo != nullptr) col_vo[s] = a;
    if (col_vss != nullptr) col_vss[s] = b;
  }
  nv->GenerateBed();
  nv->Calculate();
  for (int s = 0; s < X_D * Y_D; s++) {
    const SLOT_BUFFER_TYPE* slot = buf + static_cast<size_t>(s) * S_W * S_H;
    if (n_fin != nullptr) n_fin[s] = slot[0];
    if (fin_tzn != nullptr) {
      for (int p = 0; p < S_H; p++) {
        const bool live = p < slot[0];
        for (int k = 0; k < 3; k++)
          fin_tzn[(static_cast<size_t>(s) * S_H + p) * 3 + k] = live ? slot[(p + 1) * S_W + k] : 0;
      }
    }
  }
  if (volmass22 != nullptr) std::memcpy(volmass22, nv->vm_info.dData, sizeof(float) * 22);
  if (mat16 != nullptr) std::memcpy(mat16, nv->mat4x4.fData, sizeof(float) * 16);
  delete[] nv;
  return 0;
}

// The export tail of _TomoSh_Function_Call (Tomo_Shell2026.cpp:218-244) for
// one orientation: thread_func on it, then slotsToPxls for every pixel type
// with GetSSPixels in the eptSS entry, mat4x4 and vm_info.  counts[11] gets
// the pixel count per type; pixels receives the concatenated n x 6 int16
// records (type 0 first) up to max_pixels; returns the total count.
int ref_int3_pixels(const float* f32info, const int* i32info, const float* ypr,
                    const int* tri, const float* vtx, const float* vnrm, const float* tnrm,
                    const int* htri, const float* hvtx, const float* htnrm,
                    int ypr_index, int grid, int* counts, short* pixels, int max_pixels,
                    float* volmass22, float* mat16)
{
  S3DPrinterInfo info(const_cast<float*>(f32info), const_cast<int*>(i32info), const_cast<int*>(tri),
                      const_cast<float*>(vtx), const_cast<float*>(vnrm), const_cast<float*>(tnrm),
                      const_cast<int*>(htri), const_cast<float*>(hvtx), const_cast<float*>(htnrm), 0, 0, 0);
  STomoSh_INT3* nv = new STomoSh_INT3[1];
  prepare(nv, 1, info, grid);
  S3DPrinterInfo& pi = nv->printer_info;
  pi.yaw = ypr[ypr_index * 3 + 0];
  pi.pitch = ypr[ypr_index * 3 + 1];
  pi.roll = ypr[ypr_index * 3 + 2];
  nv->Rotate();
  nv->Pixelize();
  nv->Pairing();
  nv->GenerateBed();
  nv->Calculate();
  int total = 0;
  for (int i = 0; i < g_nPixelType; i++) {
    TPVector px = (i == static_cast<int>(enumPixelType::eptSS)) ? nv->GetSSPixels(pi.bUseExplicitSS)
                                                                : nv->slotsToPxls(enumPixelType(i));
    counts[i] = static_cast<int>(px.size());
    for (auto& q : px) {
      if (total < max_pixels) q.DumpTo(pixels + static_cast<size_t>(total) * 6);
      total++;
    }
  }
  if (volmass22 != nullptr) std::memcpy(volmass22, nv->vm_info.dData, sizeof(float) * 22);
  if (mat16 != nullptr) std::memcpy(mat16, nv->mat4x4.fData, sizeof(float) * 16);
  delete[] nv;
  return total;
}

// SMatrix4f(yaw, pitch, roll) as built by the reference (cpu_src/SMatrix4f.cpp:8-12,213-240).
float ref_int3_rotation(float yaw, float pitch, float roll, float* out16)
{
  SMatrix4f m(yaw, pitch, roll);
  std::memcpy(out16, m.fData, sizeof(float) * 16);
  return m.fData[0];
}

}  // extern "C"
