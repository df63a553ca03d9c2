/*
 * tomo_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference INT3 orientation-search path
 * (cfms-lab/Tomo_Shell2026, cfms_tomo/Tomo_Shell_vc_src/cpu_src/STomoSh_INT3.cpp
 * and friends).  Used by tests/, by __graft_entry__.smoke() and by bench.py's
 * CPU-baseline leg as the checker.  The product library never links it.
 *
 * Parity of this restatement is pinned against the reference engine itself,
 * compiled from the reference sources into oracle/_ref/libtomo_ref.so, and
 * against golden fixtures generated from it (tests/golden/).
 */
#ifndef TOMO_ORACLE_H
#define TOMO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Rotation used for one orientation: SMatrix4f::YPR (cpu_src/SMatrix4f.cpp:213-240).
 * Writes the 3x3 block row-major. */
void tomo_oracle_rotation(float yaw, float pitch, float roll, float R9[9]);

/* Shadow threshold FLOAT32(-1. * ::sin(theta_c)) (cpu_src/STomoSh_INT3.cpp:756). */
float tomo_oracle_threshold(float theta_c);

/* Mass model STomoVolMassInfo::VolToMass (cpu_src/STomoVolMassInfo.cpp:42-80).
 * vm22 holds the 22-float vm_info block with Va..Vtc, Vss, Vo, Vbed filled in;
 * the mass fields are written. */
void tomo_oracle_vol_to_mass(const float* f32info12, const int32_t* i32info11, float* vm22);

/* Whole sweep.  Returns the reference optID (_find1stOptimal,
 * Tomo_Shell2026.cpp:89-97) or a negative error code:
 *   -1 bad arguments, -2 out of memory, -3 a slot index fell outside the grid.
 * grid: square slot grid edge (0 = 256, the reference default).
 * Outputs are [nYPR] and may be NULL. */
int tomo_oracle_sweep(const float* f32info12, const int32_t* i32info11, const float* ypr,
                      const int32_t* tri, const float* vtx, const float* vtx_nrm,
                      int grid, int n_threads,
                      float* Mo, float* Mss, float* Vtc, float* VoF, float* VssF,
                      int64_t* Vo64, int64_t* Vss64, int64_t* Vtc64,
                      int64_t* n_entries, int64_t* n_columns);

/* One orientation with per-column dumps, same layout as the reference driver
 * (oracle/ref/ref_driver.cpp ref_int3_columns).  Any output may be NULL.
 *   n_vox[g*g], vox_zn[g*g*64*2]  slot lists right after voxelization
 *   n_fin[g*g], fin_tzn[g*g*64*3] slot lists after pairing and bed
 *   col_vo, col_vss, col_vtc      per-column values
 *   vm22                          vm_info after Calculate, mat16 the 4x4 */
int tomo_oracle_columns(const float* f32info12, const int32_t* i32info11, const float* ypr,
                        const int32_t* tri, const float* vtx, const float* vtx_nrm,
                        int ypr_index, int grid,
                        int32_t* n_vox, int16_t* vox_zn, int32_t* n_fin, int16_t* fin_tzn,
                        int32_t* col_vo, int32_t* col_vss, int32_t* col_vtc,
                        float* vm22, float* mat16);

#ifdef __cplusplus
}
#endif
#endif
