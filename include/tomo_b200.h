/*
 * tomo_b200.h -- C-ABI of libtomo_b200.so, the B200 (sm_100a) orientation
 * search of cfms-lab/Tomo_Shell2026.
 *
 * The first block is a drop-in for the reference DLL exports
 * (cfms_tomo/Tomo_Shell_vc_src/Tomo_Shell2026.h:19-35) as bound by the
 * reference Python surface through ctypes (cfms_tomo/tomo_dll_interface.py:23-43,
 * cfms_tomo/shell_test/tomoSh_Cpp.py:67-120).  Same names, argument order and
 * meaning; MESH_ELE_ID_TYPE is int32, FLOAT32 is float, INT16 is short.
 * Differences: errors return negative codes instead of terminating the
 * process, results are exact (int64 totals are exported next to the float
 * ones), and the library never calls cudaDeviceReset.
 *
 * All buffers returned by getters are owned by the library and stay valid
 * until the next TomoSh_CUDA call or OnDestroy.  Calls are serialised by an
 * internal lock; one process drives one GPU (the current CUDA device).
 */
#ifndef TOMO_B200_H
#define TOMO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* error codes (returned by TomoSh_CUDA and the tomo* calls; 0 or an index on success) */
#define TOMO_ERR_ARG (-1)       /* bad argument (null pointer, negative size, index out of range) */
#define TOMO_ERR_CUDA (-2)      /* CUDA runtime error, see tomoGetLastErrorString */
#define TOMO_ERR_CAPACITY (-3)  /* a fixed capacity was exceeded (grid, shared-memory column strip) */

/* ---- reference-compatible exports ---------------------------------------- */

/* Exhaustive orientation search.  Replaces TomoSh_CUDA / TomoSh_INT3
 * (Tomo_Shell2026.h:33-35, Tomo_Shell2026.cpp:119-248,257-260,328-378).
 *   f32info[12]  dVoxel, theta_c, surface_area, wall_thickness, Fcore, Fclad,
 *                Fss, Css, PLA_density, BedInnerBound, BedOuterBound, BedThickness
 *                (S3DPrinterInfo.h:42-47)
 *   i32info[11]  bVerbose, bUseExplicitSS, bShellMesh, nVoxel, nTri, nVtx, nYPR,
 *                nHullTri, nHullVtx, BedType, ShellThickness*1000 (S3DPrinterInfo.cpp:132-144)
 *   YPR[nYPR*3]  yaw, pitch, roll in radians
 *   tri[nTri*3], vtx[nVtx*3], vtx_nrm[nVtx*3]  mesh; tri_nrm and the convex
 *                hull arrays are accepted and unused (the INT3 arithmetic does
 *                not read them).
 * Returns optID = first index of the strictly smallest Mss starting from
 * 1e5 (_find1stOptimal, Tomo_Shell2026.cpp:89-97), or a negative error. */
int TomoSh_CUDA(float* f32info, int* i32info, float* YPR, int* tri, float* vtx, float* vtx_nrm, float* tri_nrm,
                int* chull_tri, float* chull_vtx, float* chull_trinrm);

/* Same call under the reference's CPU-engine name (Tomo_Shell2026.h:33,
 * Tomo_Shell2026.cpp:257-260): the reference INT3 results, computed on the GPU. */
int TomoSh_INT3(float* f32info, int* i32info, float* YPR, int* tri, float* vtx, float* vtx_nrm, float* tri_nrm,
                int* chull_tri, float* chull_vtx, float* chull_trinrm);

/* getMss / getMo / getVtc: [nYPR] float32 (Tomo_Shell2026.h:21-23). */
float* getMss(void);
float* getMo(void);
float* getVtc(void);
/* 22-float vm_info of the best orientation (Tomo_Shell2026.h:24, STomoVolMassInfo.h:19-33). */
float* getVolMassInfo(void);
/* 4x4 transform of the best orientation (Tomo_Shell2026.h:25, STomoSh_Base.cpp:155-167). */
float* getMat4x4(void);
/* Render pixels of the best orientation by enumPixelType (Tomo_Shell2026.h:19-20);
 * n x 6 int16 (x, y, z, nx, ny, nz). */
int getnData2i(short type);
short* getpData2i(short type);
/* Frees every library buffer and the device work memory (Tomo_Shell2026.h:29). */
void OnDestroy(void);

/* ---- additions -------------------------------------------------------------- */

/* Exact per-orientation totals [nYPR] of the last call: sum of per-column
 * Vo / Vss / Vtc in int64 (the reference keeps them in float32,
 * STomoVolMassInfo.h:24-31; its own debug accumulator is int64,
 * STomoSh_INT3.cpp:129-170). */
const long long* getVo64(void);
const long long* getVss64(void);
const long long* getVtc64(void);

int tomoGetLastError(void);
const char* tomoGetLastErrorString(void);

/* Host-side pieces, exported so tests can pin them to the reference:
 * rotation of SMatrix4f::YPR (SMatrix4f.cpp:213-240), 3x3 row-major;
 * shadow threshold of STomoSh_INT3.cpp:756; VolToMass of STomoVolMassInfo.cpp:42-80. */
void tomoRotation(float yaw, float pitch, float roll, float* out9);
float tomoShadowThreshold(float theta_c);
void tomoVolToMass(const float* f32info, const int* i32info, float* vm22);

/* Tuning / test hooks. */
#define TOMO_OPT_BATCH 1        /* orientations per device batch (default 256) */
#define TOMO_OPT_STRIP_H 2      /* force strip height 1, 2, 4 or 8 (0 = automatic) */
#define TOMO_OPT_FORCE_SAFE 3   /* 1 = evaluate every orientation in safe mode */
#define TOMO_OPT_NORMAL_SMEM 4  /* shared-memory bytes of a normal strip CTA (0 = the largest that keeps four per SM, ~55 KB) */
#define TOMO_OPT_EXPORT 5       /* 0 = skip the best orientation's pixel export (default 1) */
#define TOMO_OPT_ADAPTIVE 6     /* 0 = keep the planned strip budget even when early batches overflow (default 1) */
#define TOMO_OPT_PROPOSAL 7     /* tomoSurrogateSearch proposals: 0 = the trained network (default), 1 = bilinear
                                   interpolation of the exact coarse values (the search without the network),
                                   2 = the mean of the two */
#define TOMO_OPT_FOLD_LIMIT 8   /* largest |column value| a packed 16-bit fold record holds (1..32767, default 32767);
                                   larger values go through the batch's escape table.  Lower only to test that table */
int tomoSetOption(int key, int value);

/* out[0..8] = grid edge, strip height, strips, entry capacity, orientations re-run
 * with a large strip capacity, nYPR, batch, orientations re-run in safe mode,
 * orientations re-run with first-come priorities (a column past the 63 cap) --
 * of the last TomoSh_CUDA-style sweep, zero before the first; out[9..11] = the
 * same three re-run counts (large capacity, priorities, safe mode) of the last
 * tomoSweepStatic call.  Returns TOMO_ERR_ARG only for a null `out`. */
int tomoGetStats(long long* out, int n);

/* Per-orientation results of the last sweep; any pointer may be null. */
int tomoGetResults(long long* vo64, long long* vss64, long long* vtc64, float* vof, float* vssf, float* vtcf,
                   int* nbed, int* flags, long long* entries, long long* columns);

/* Split form of TomoSh_CUDA: upload the mesh and orientations once, run the
 * device sweep any number of times with the inputs resident in device memory
 * (optionally bracketed by caller-created cudaEvent_t handles; kernel_ms
 * receives the elapsed device time), then finish on the host. */
int tomoPrepare(const float* f32info, const int* i32info, const float* YPR, const int* tri, const float* vtx,
                const float* vtx_nrm);
int tomoSweepDevice(void* ev_start, void* ev_stop, float* kernel_ms);
int tomoFinish(float* Mo, float* Mss, float* Vtc);

/* Launch accounting.  Kernel kinds, in order: reset, rotate, bin_count,
 * bin_scan, bin_fill, strip, bed, fold, strip re-runs.  tomoProfile(enable, reset) turns
 * per-launch CUDA-event timing on or off (events are recorded on the stream
 * each kernel is launched on) and optionally clears the log;
 * tomoGetKernelLog fills launches / total ms / timed launches per kind and
 * returns the number of kinds. */
int tomoProfile(int enable, int reset);
int tomoGetKernelLog(long long* launches, double* ms, long long* timed, int n);

/* Read-bandwidth probe (no counterpart in the reference; a measurement aid):
 * one untimed pass, then `reps` timed passes of a kernel that reads the
 * caller's device buffer (16-byte aligned, `bytes` long) through L2;
 * *ms_out = device time of the timed passes.  A buffer well inside the
 * 126 MB L2 gives the L2 read bandwidth; a larger one the HBM read bandwidth. */
int tomoProbeReadBandwidth(const void* dev_buf, long long bytes, int reps, float* ms_out);

/* Slot grid edge G of the prepared mesh (slot id = x * G + y). */
int tomoGridSize(void);

/* One orientation of the prepared sweep with a dense per-column dump (parity
 * tests; no reference counterpart -- the reference writes comparable CSV
 * dumps behind TOMO_DEBUG_PAIR_OUTPUT, STomoSh_INT3.cpp:172-235).
 *   cols8[G*G*8]    n_distinct, n_final, vo, vss, tc, last_z, last_type, bed flags
 *   keys64[G*G*64]  kept (z, nz) keys, (z+32768)<<16 | (nz+32768), in column order
 *   types64[G*G*64] their type bits after pairing
 * Returns the orientation's status flags (>= 0) or a negative error. */
int tomoColumnDump(int ypr_index, int safe_mode, int* cols8, unsigned* keys64, short* types64);

/* ---- multi-mesh batch (the additive TomoSh_CUDA_Batch export; no reference
 * counterpart, the reference front-end loops over parts calling TomoSh_CUDA,
 * cfms_tomo/__init__.py:26-30).  Each argument is an array of n_mesh pointers
 * to that mesh's TomoSh_CUDA argument; meshes may differ in triangle count,
 * printer options and orientation list.  tomoBatchPrepare uploads every mesh
 * and picks each size class's strip configuration by timing candidates
 * (autotuner); tomoBatchRun sweeps all meshes -- with use_graph, as one CUDA
 * graph captured on the first run and replayed after -- re-runs flagged
 * orientations per mesh and leaves per-mesh results equal to TomoSh_CUDA on
 * that mesh alone; device_ms receives the time on the library's stream from
 * the start of the sweep until every mesh is resolved (re-runs included).
 * tomoBatchResults copies mesh `mesh`'s per-orientation results (any pointer
 * may be null) and returns its optID.  TomoSh_CUDA_Batch = prepare + run with
 * the graph + optIDs[n_mesh]. */
int tomoBatchPrepare(int n_mesh, const float* const* f32info, const int* const* i32info, const float* const* YPR,
                     const int* const* tri, const float* const* vtx, const float* const* vtx_nrm);
int tomoBatchRun(int use_graph, float* device_ms);
int tomoBatchResults(int mesh, float* Mo, float* Mss, float* Vtc, long long* vo64, long long* vss64, long long* vtc64);
int TomoSh_CUDA_Batch(int n_mesh, const float* const* f32info, const int* const* i32info, const float* const* YPR,
                      const int* const* tri, const float* const* vtx, const float* const* vtx_nrm, int* optIDs);
/* out[0..7] = meshes, orientations, graph nodes, kernels per graph launch,
 * size classes tuned by the last prepare, size classes tuned so far,
 * orientations re-run, time of the last run in microseconds (sweep and
 * re-runs, as device_ms), time of its sweep alone (the graph replay) */
int tomoBatchStats(long long* out, int n);
/* out4 = orientations per batch, normal-CTA shared-memory budget (0 = four CTAs per SM),
 * strip height, slot-grid edge chosen for mesh `mesh` */
int tomoBatchConfig(int mesh, int* out4);
/* The TomoSh_CUDA tail for mesh `mesh` of the last tomoBatchRun: the getters
 * (getMss, getMo, getVtc, getVolMassInfo, getMat4x4, getnData2i, getpData2i,
 * getVo64 ...) then return that mesh's results as if TomoSh_CUDA had run on
 * it alone.  Returns its optID. */
int tomoBatchExport(int mesh);
/* key 1: autotune on/off (default 1); key 2: autotune sample orientations (default 512) */
int tomoBatchSetOption(int key, int value);
void tomoBatchRelease(void);

/* ---- learned-proposal search (no reference counterpart) -------------------
 * The surrogate network: an FP32 MLP [sin yaw, cos yaw, sin pitch, cos pitch]
 * -> 128 -> 128 -> 128 -> 1 (tanh hidden units, linear output) trained with
 * mean squared error and Adam by the library's own CUDA kernels.  Host
 * arrays: x[n][4] features, y[n] targets.  Parameters are one flat float
 * vector (per layer weights [in][out] row-major, then biases; 33,793 in all).
 *   tomoMlpInit      seeded initialisation, Adam state cleared; returns the parameter count
 *   tomoMlpParams    copy the parameters out (get) and/or in (set; clears Adam state)
 *   tomoMlpGrad      forward + backward on (x, y): flat gradient and loss
 *   tomoMlpAdam      one Adam step from the last gradient
 *   tomoMlpFit       steps x (gradient + Adam) on (x, y); loss of the last step
 *   tomoMlpPredict   out[n] = network(x) */
int tomoMlpInit(int seed);
int tomoMlpParams(float* get, const float* set);
int tomoMlpGrad(const float* x, const float* y, int n, float* grad, float* loss);
int tomoMlpAdam(float lr);
int tomoMlpFit(const float* x, const float* y, int n, int steps, float lr, float* loss);
int tomoMlpPredict(const float* x, int n, float* out);

/* Learned-proposal search over a YPR grid laid out [n_pitch][n_yaw] (yaw
 * fastest; n_yaw * n_pitch = Int32Info[6]).  The exact kernels evaluate the
 * coarse points (both grid indices multiples of `stride`); the network is
 * trained on their exact Vss, except a seeded `holdout` share kept to measure
 * its error; it ranks the cell x cell blocks of the grid by their smallest
 * predicted Vss and the top_k blocks are evaluated exactly.  Then, round
 * after round, every block whose smallest prediction minus margin x (largest
 * error seen on any evaluated point not trained on) is at or below the best
 * exact Vss is evaluated too.  The search falls back to the exhaustive sweep
 * when that would exceed max_eval evaluated orientations (0 = nYPR / 5), when
 * the mean relative error of the untrained points exceeds `gate`, or with a
 * bed (Mss is then not a function of Vss alone).
 * iparams = {stride, cell, top_k, train_steps, seed, max_eval},
 * fparams = {learning_rate, gate, margin, holdout, log_scale}: with
 * log_scale > 0 the network learns log1p((Vss - min) / s), s = log_scale x
 * (median - min) of its training Vss, instead of Vss.  Returns optID
 * (_find1stOptimal over the evaluated orientations, grid order).
 * Mss_out[nYPR]: exact Mss where evaluated, NaN elsewhere; pred_out[nYPR]:
 * predicted Vss (either may be null).  stats[12] = evaluated orientations,
 * fell back (0/1), mean relative error, max abs error, final training loss,
 * seconds total / exact sweeps / training / prediction, blocks refined,
 * expansion rounds, coarse points. */
int tomoSurrogateSearch(const float* f32info, const int* i32info, const float* YPR, const int* tri, const float* vtx,
                        const float* vtx_nrm, int n_yaw, int n_pitch, const int* iparams, const float* fparams,
                        float* Mss_out, float* pred_out, double* stats);

/* Allocation-free form of TomoSh_CUDA for small meshes.  No counterpart in the
 * reference.  Same inputs as TomoSh_CUDA; Mo, Mss and Vtc are caller-owned
 * host arrays of nYPR floats that receive what getMo/getMss/getVtc return
 * after TomoSh_CUDA, and the return value is optID (or a negative error).
 * The render pixels, vm_info and mat4x4 are not produced.
 *   - allocates nothing: device scratch is one file-scope 8 MiB __device__
 *     array per device, host staging is file-scope arrays; no cudaMalloc,
 *     cudaFree or allocating library routine is called;
 *   - limits: at most 16384 triangles and 16384 vertices, and a footprint
 *     within the reference's 256 x 256 slot grid; larger inputs return
 *     TOMO_ERR_CAPACITY with the limit in tomoGetLastErrorString();
 *   - the scratch's device address is looked up with cudaGetSymbolAddress the
 *     first time a device is used (with that device current), so make the first
 *     call on each device before any stream capture begins; the address is kept
 *     for the life of the process, so no cudaDeviceReset (which unloads this
 *     library's device code) may come between two calls on that device;
 *   - nothing has to start at zero: each batch clears what its kernels
 *     accumulate into (the bed pixel counts by cudaMemsetAsync, the rest in
 *     the first kernel);
 *   - the scratch is shared by every call on a device, so two calls whose
 *     device work overlapped would race on it; the call holds the library's
 *     lock and synchronizes `stream` before it returns -- error returns
 *     included, once any device work was issued -- so calls from several
 *     host threads run one after another;
 *   - orientations that a strip cannot resolve alone are re-run in the same
 *     configurations as TomoSh_CUDA (large capacity, first-come priorities,
 *     safe mode); tomoGetStats out[9..11] counts them for the last call;
 *   - work is issued on `stream` (a cudaStream_t; null = the legacy default
 *     stream), orientations four at a time. */
int tomoSweepStatic(const float* f32info, const int* i32info, const float* YPR, const int* tri, const float* vtx,
                    const float* vtx_nrm, float* Mo, float* Mss, float* Vtc, void* stream);

#ifdef __cplusplus
}
#endif
#endif
