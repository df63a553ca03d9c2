/*
 * tomo_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference INT3 orientation search
 * (cfms-lab/Tomo_Shell2026, cfms_tomo/Tomo_Shell_vc_src).  It exists to check
 * the CUDA implementation: tests/, __graft_entry__.smoke() and the bench's
 * CPU-baseline leg call it; the product library never does.
 *
 * Parity pin: every function below is checked bit-for-bit against the
 * reference engine compiled from its own sources (oracle/_ref/libtomo_ref.so,
 * recipe oracle/build.py) and against the golden fixtures generated from it
 * (tests/golden/make_golden.py).
 *
 * All float arithmetic is single precision with one rounding per operation
 * (built with -ffp-contract=off, no fast-math), in the reference's operation
 * order; the three places where the reference widens to double are kept.
 * Reference file references are relative to cfms_tomo/Tomo_Shell_vc_src.
 */
#define _POSIX_C_SOURCE 200809L
#include "tomo_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---- constants (Tomo_types.h:38-40,72-82; STomoVoxelSpaceInfo.cpp:47-51) ---- */
#define MARGIN 0.001f          /* g_fMARGIN */
#define NORMAL_FACTOR 1000.0f  /* g_fNORMALFACTOR */
#define ROWS 64                /* nSlotCapacityHeight with _USE_BRIEF_SLOT_PAIRING */
#define CAP (ROWS - 1)         /* pixels a slot can hold (SetBit rejects at count >= 63) */

enum {
  T_AL = 1, T_BE = 2, T_SSB = 4, T_SSA = 8, T_SS = 16, T_BED = 32,
  T_VO = 64, T_VSS = 128, T_TC = 256, T_NVB = 512, T_NVA = 1024
};
enum { BED_NONE = 0, BED_BRIM = 1, BED_RAFT = 2, BED_SKIRT = 3 };

/* ---- printer info (S3DPrinterInfo.h:42-47, S3DPrinterInfo.cpp:130-144) ---- */
typedef struct {
  float dVoxel, theta_c, surface_area, wall, Fcore, Fclad, Fss, Css, rho;
  float bed_inner, bed_outer, bed_thickness;
  int explicit_ss, shell, n_tri, n_vtx, n_ypr, bed_type;
  float shell_thickness;
} params_t;

static void read_params(const float* f, const int32_t* i, params_t* p)
{
  p->dVoxel = f[0]; p->theta_c = f[1]; p->surface_area = f[2]; p->wall = f[3];
  p->Fcore = f[4]; p->Fclad = f[5]; p->Fss = f[6]; p->Css = f[7]; p->rho = f[8];
  p->bed_inner = f[9]; p->bed_outer = f[10]; p->bed_thickness = f[11];
  /* (_int32_x11[k] > g_fMARGIN) compares int with float (S3DPrinterInfo.cpp:132-134) */
  p->explicit_ss = ((float)i[1] > MARGIN);
  p->shell = ((float)i[2] > MARGIN);
  p->shell_thickness = (float)i[10] * 0.001f;
  p->n_tri = i[4]; p->n_vtx = i[5]; p->n_ypr = i[6]; p->bed_type = i[9];
}

/* ---- rotation: SMatrix4f::YPR (SMatrix4f.cpp:213-240) ---- */
void tomo_oracle_rotation(float ga, float be, float al, float R[9])
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

/* SMatrix4f::Dot (SMatrix4f.cpp:242-262): sequential +=, homogeneous column
 * of the pure rotation is zero, so the last term adds 0*1. */
static inline void dot3(const float R[9], const float a[3], float out[3])
{
  const float t0 = a[0], t1 = a[1], t2 = a[2];
  for (int r = 0; r < 3; r++) {
    float s = R[r * 3 + 0] * t0;
    s += R[r * 3 + 1] * t1;
    s += R[r * 3 + 2] * t2;
    s += 0.0f * 1.0f;
    out[r] = s;
  }
}

float tomo_oracle_threshold(float theta_c)
{
  return (float)(-1.0 * (double)sinf(theta_c)); /* STomoSh_INT3.cpp:756 (float overload) */
}

/* ---- per-thread workspace ---- */
typedef struct {
  int g;              /* grid edge; slot id = x*g + y (STomoVoxelSpaceInfo.cpp:242) */
  uint8_t* cnt;       /* pixels per slot */
  int16_t* z;         /* [g*g*ROWS] */
  int16_t* nz;
  int16_t* type;
  int32_t* dirty;     /* slots in the order they became non-empty */
  int n_dirty;
  int cap_dirty;
  float* vtx1;        /* rotated + translated vertices */
  float* nrm1;        /* rotated vertex normals */
  int error;
} ws_t;

static int ws_init(ws_t* w, int g, int n_vtx)
{
  memset(w, 0, sizeof(*w));
  w->g = g;
  size_t ns = (size_t)g * g;
  w->cnt = calloc(ns, 1);
  w->z = calloc(ns * ROWS, sizeof(int16_t));
  w->nz = calloc(ns * ROWS, sizeof(int16_t));
  w->type = calloc(ns * ROWS, sizeof(int16_t));
  w->cap_dirty = 1024;
  w->dirty = malloc(sizeof(int32_t) * (size_t)w->cap_dirty);
  w->vtx1 = malloc(sizeof(float) * 3 * (size_t)(n_vtx > 0 ? n_vtx : 1));
  w->nrm1 = malloc(sizeof(float) * 3 * (size_t)(n_vtx > 0 ? n_vtx : 1));
  return (w->cnt && w->z && w->nz && w->type && w->dirty && w->vtx1 && w->nrm1) ? 0 : -2;
}

static void ws_free(ws_t* w)
{
  free(w->cnt); free(w->z); free(w->nz); free(w->type); free(w->dirty);
  free(w->vtx1); free(w->nrm1);
}

/* ClearDirtySlots (STomoVoxelSpaceInfo.cpp:62-80): the reference zeroes the
 * slots touched by the previous orientation. */
static void ws_clear(ws_t* w)
{
  for (int i = 0; i < w->n_dirty; i++) {
    size_t s = (size_t)w->dirty[i];
    w->cnt[s] = 0;
    memset(w->z + s * ROWS, 0, ROWS * sizeof(int16_t));
    memset(w->nz + s * ROWS, 0, ROWS * sizeof(int16_t));
    memset(w->type + s * ROWS, 0, ROWS * sizeof(int16_t));
  }
  w->n_dirty = 0;
  w->error = 0;
}

static void mark_dirty(ws_t* w, int32_t s)
{
  if (w->n_dirty == w->cap_dirty) {
    int nc = w->cap_dirty * 2;
    int32_t* nd = realloc(w->dirty, sizeof(int32_t) * (size_t)nc);
    if (!nd) { w->error = -2; return; }
    w->dirty = nd; w->cap_dirty = nc;
  }
  w->dirty[w->n_dirty++] = s;
}

/* SetBit (STomoVoxelSpaceInfo.cpp:175-229): truncating casts for slot, z and
 * nz; exact (z, nz) dedup; first-come append; silent drop at 63 pixels. */
static void set_bit(ws_t* w, const float pxl[3], const float nrm[3], int type_byte)
{
  const int sx = (int)pxl[0];
  const int sy = (int)pxl[1];
  if (sx < 0 || sy < 0 || sx >= w->g || sy >= w->g) { w->error = -3; return; }
  const int16_t pz = (int16_t)(int)pxl[2];
  const int16_t pnz = (int16_t)(int)(nrm[2] * NORMAL_FACTOR);
  const int32_t s = sx * w->g + sy;
  const size_t base = (size_t)s * ROWS;
  const int n = w->cnt[s];
  int id = -1;
  for (int p = 0; p < n; p++) {
    if (w->z[base + p] == pz && w->nz[base + p] == pnz) { id = p; break; }
  }
  if (id < 0) {
    if (n >= CAP) return;
    if (n == 0) mark_dirty(w, s);
    id = n;
    w->cnt[s] = (uint8_t)(n + 1);
  }
  w->type[base + id] |= (int16_t)type_byte;
  w->z[base + id] = pz;
  w->nz[base + id] = pnz;
}

/* _getBaryCoord (Tomo_types.cpp:86-115).  u is formed in double and the
 * upper bounds are compared in double, as in the reference. */
static int bary(const float p[3], const float a[3], const float b[3], const float c[3],
                float* u, float* v, float* w)
{
  const float e0x = b[0] - a[0], e0y = b[1] - a[1];
  const float e1x = c[0] - a[0], e1y = c[1] - a[1];
  const float e2x = p[0] - a[0], e2y = p[1] - a[1];
  const float d00 = e0x * e0x + e0y * e0y + 0.0f * 0.0f;
  const float d01 = e0x * e1x + e0y * e1y + 0.0f * 0.0f;
  const float d11 = e1x * e1x + e1y * e1y + 0.0f * 0.0f;
  const float d20 = e2x * e0x + e2y * e0y + 0.0f * 0.0f;
  const float d21 = e2x * e1x + e2y * e1y + 0.0f * 0.0f;
  const float denom = d00 * d11 - d01 * d01;
  const float adenom = ((double)denom >= 0.) ? denom : -denom;
  if (adenom > MARGIN) {
    const float vv = (d11 * d20 - d01 * d21) / denom;
    const float ww = (d00 * d21 - d01 * d20) / denom;
    const float uu = (float)(1.0 - (double)vv - (double)ww);
    if (uu >= -MARGIN && vv >= -MARGIN && (double)vv <= 1. + (double)MARGIN &&
        (double)(uu + vv) <= 1. + (double)MARGIN) {
      *u = uu; *v = vv; *w = ww;
      return 1;
    }
  }
  *u = -1.f; *v = -1.f; *w = -1.f;
  return 0;
}

/* _bary_product (Tomo_types.cpp:75-84) */
static inline void bary_product(const float p0[3], const float p1[3], const float p2[3],
                                float u, float v, float w, float out[3])
{
  for (int i = 0; i < 3; i++) out[i] = p0[i] * u + p1[i] * v + p2[i] * w;
}

/* triVoxel (STomoSh_INT3.cpp:1138-1209) */
static int tri_voxel(ws_t* w, const params_t* P, const float* _v0, const float* _v1, const float* _v2,
                     const float* n0, const float* n1, const float* n2)
{
  float v0[3], v1[3], v2[3];
  for (int i = 0; i < 3; i++) {
    v0[i] = _v0[i] + MARGIN;
    v1[i] = _v1[i] + MARGIN;
    v2[i] = _v2[i] + MARGIN;
  }
#define FMIN(a, b) (((a) <= (b)) ? (a) : (b))
#define FMAX(a, b) (((a) >= (b)) ? (a) : (b))
  const int x0 = (int)FMIN(FMIN(v0[0], v1[0]), v2[0]);
  const int y0 = (int)FMIN(FMIN(v0[1], v1[1]), v2[1]);
  const int x1 = (int)FMAX(FMAX(v0[0], v1[0]), v2[0]);
  const int y1 = (int)FMAX(FMAX(v0[1], v1[1]), v2[1]);
  const float half = P->dVoxel * 0.5f;
  const float shell_off = (float)(int)(P->shell_thickness + 0.999f);
  const int twin = P->shell && P->shell_thickness > MARGIN;
  float center[3] = {0.f, 0.f, half};
  int hits = 0;
  for (int x = x0; x <= x1; x++) {
    center[0] = ((float)x + MARGIN) + half;
    for (int y = y0; y <= y1; y++) {
      center[1] = ((float)y + MARGIN) + half;
      float u, v, ww;
      if (bary(center, v0, v1, v2, &u, &v, &ww)) {
        float pxl[3], nrm[3];
        bary_product(v0, v1, v2, u, v, ww, pxl);
        bary_product(n0, n1, n2, u, v, ww, nrm);
        set_bit(w, pxl, nrm, 0);
        hits++;
        if (twin) {
          pxl[2] += (nrm[2] >= 0) ? -shell_off : shell_off;
          nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
          set_bit(w, pxl, nrm, 0);
          hits++;
        }
      }
    }
  }
  if (hits == 0) {
    float c[3];
    for (int i = 0; i < 3; i++) c[i] = (_v0[i] + _v1[i] + _v2[i]) * 0.333333f + MARGIN;
    set_bit(w, c, n0, 0);
    if (twin) {
      float sc[3] = {c[0], c[1], c[2]};
      float sn[3] = {-n0[0], -n0[1], -n0[2]};
      sc[2] += (n0[2] >= 0) ? -shell_off : shell_off;
      set_bit(w, sc, sn, 0);
    }
  }
  return hits;
#undef FMIN
#undef FMAX
}

/* STomoSh_Base::Rotate (STomoSh_Base.cpp:45-129) with STomoAABB3Df::Set /
 * GetCenter (STomoAABB3Df.cpp:58-72). */
static void rotate(ws_t* w, const params_t* P, const float* vtx, const float* vnrm,
                   float yaw, float pitch, float roll, float mat16[16])
{
  const int nV = P->n_vtx;
  float mn[3] = {1e5f, 1e5f, 1e5f}, mx[3] = {-1e5f, -1e5f, -1e5f};
  for (int v = 0; v < nV; v++)
    for (int i = 0; i < 3; i++) {
      const float d = vtx[v * 3 + i];
      mn[i] = (mn[i] <= d) ? mn[i] : d;
      mx[i] = (mx[i] >= d) ? mx[i] : d;
    }
  float c[3];
  for (int i = 0; i < 3; i++) c[i] = (float)((double)(mn[i] + mx[i]) * 0.5);
  float R[9];
  tomo_oracle_rotation(yaw, pitch, roll, R);
  for (int v = 0; v < nV; v++) {
    float t[3] = {vtx[v * 3 + 0] - c[0], vtx[v * 3 + 1] - c[1], vtx[v * 3 + 2] - c[2]};
    dot3(R, t, w->vtx1 + v * 3);
    dot3(R, vnrm + v * 3, w->nrm1 + v * 3);
  }
  float rmn[3] = {1e5f, 1e5f, 1e5f};
  for (int v = 0; v < nV; v++)
    for (int i = 0; i < 3; i++) {
      const float d = w->vtx1[v * 3 + i];
      rmn[i] = (rmn[i] <= d) ? rmn[i] : d;
    }
  const float dx = rmn[0] - P->bed_outer, dy = rmn[1] - P->bed_outer, dz = rmn[2];
  for (int v = 0; v < nV; v++) {
    w->vtx1[v * 3 + 0] -= dx;
    w->vtx1[v * 3 + 1] -= dy;
    w->vtx1[v * 3 + 2] -= dz;
  }
  if (mat16) {
    const float m = -c[0], n = -c[1], o = -c[2];
    const float tu = -dx, tv = -dy, tw = -dz;
    memset(mat16, 0, 16 * sizeof(float));
    for (int r = 0; r < 3; r++)
      for (int k = 0; k < 3; k++) mat16[r * 4 + k] = R[r * 3 + k];
    mat16[15] = 1.f;
    mat16[3] = tu + R[0] * m + R[1] * n + R[2] * o;
    mat16[7] = tv + R[3] * m + R[4] * n + R[5] * o;
    mat16[11] = tw + R[6] * m + R[7] * n + R[8] * o;
  }
}

/* Pixelize (STomoSh_INT3.cpp:285-364): triangles in index order. */
static void pixelize(ws_t* w, const params_t* P, const int32_t* tri)
{
  ws_clear(w);
  for (int t = 0; t < P->n_tri && w->error == 0; t++) {
    const int a = tri[t * 3 + 0], b = tri[t * 3 + 1], c = tri[t * 3 + 2];
    tri_voxel(w, P, w->vtx1 + a * 3, w->vtx1 + b * 3, w->vtx1 + c * 3,
              w->nrm1 + a * 3, w->nrm1 + b * 3, w->nrm1 + c * 3);
  }
}

static int cmp_i32(const void* a, const void* b)
{
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* One column through vslotPair's brief branch (STomoSh_INT3.cpp:1041-1062):
 *   sortSlotByZ  (:398-446)  z descending, equal z by nz descending -- keys
 *                            are unique after SetBit's dedup, so this is a
 *                            total order;
 *   splitAlBe    (:493-513)  alpha if nz*1000.f > 0.01, beta if < -0.01;
 *   matchAlBePairBriefly (:583-611) keep alpha opening / beta closing a pair,
 *                            zero the type of any other alpha or beta;
 *   createVoPixels (:934-960), createShadowBriefly (:749-812),
 *   createTCPixels (:734-747, implicit mode), createVss_* (:962-1025).
 * The stages are left-to-right scans whose state at row p depends only on
 * rows <= p, so they are evaluated in one pass here.  Rows of the slot are
 * rewritten in sorted order with their final types; sentinel rows are
 * appended.  Returns the new pixel count. */
static int pair_column(int16_t* z, int16_t* nz, int16_t* type, int n, const params_t* P, float thr,
                       int32_t* vo, int32_t* vss, int32_t* tc_out)
{
  /* insertion sort on the (z, nz) key, descending */
  for (int i = 1; i < n; i++) {
    const int16_t kz = z[i], kn = nz[i], kt = type[i];
    int j = i - 1;
    while (j >= 0 && (z[j] < kz || (z[j] == kz && nz[j] < kn))) {
      z[j + 1] = z[j]; nz[j + 1] = nz[j]; type[j + 1] = type[j];
      j--;
    }
    z[j + 1] = kz; nz[j + 1] = kn; type[j + 1] = kt;
  }
  int started = 0, ex = 0, im = 0, tc_done = 0;
  int32_t al = 0, bes = 0, ssb = 0, ssa = 0, tc = 0, nvb = 0, nva = 0;
  for (int p = 0; p < n; p++) {
    int t = type[p];
    const float fnz = (float)nz[p] * NORMAL_FACTOR;
    if ((double)fnz > (double)MARGIN * 10.) t |= T_AL;
    else if ((double)fnz < (double)MARGIN * -10.) t |= T_BE;
    if (!started && t == T_AL) started = 1;
    else if (started && t == T_BE) started = 0;
    else if (t == T_AL || t == T_BE) t = 0;
    if (t & T_BE) {
      const float pn = (float)nz[p] / NORMAL_FACTOR;
      if (pn < MARGIN) {
        if (!ex && pn < thr) { t |= T_SSB; ex = 1; }
        if (!im && pn > thr) { t |= T_NVB; im = 1; }
      }
    } else if (t & T_AL) {
      if (ex) { t |= T_SSA; ex = 0; }
      if (im) { t |= T_NVA; im = 0; }
    }
    if (!P->explicit_ss && !tc_done && (t & T_AL)) { t |= T_TC; tc_done = 1; }
    type[p] = (int16_t)t;
    if (t & T_AL) {
      al += z[p];
      if (t & T_TC) tc += z[p];
      if (t & T_NVA) nva += z[p];
    } else if (t & T_BE) {
      bes += z[p];
      if (t & T_NVB) nvb += z[p];
    }
    if (t & T_SSB) ssb += z[p];
    else if (t & T_SSA) ssa += z[p];
  }
  /* unclosed shadows get a floor sentinel at z = 0 while room remains
   * (STomoSh_INT3.cpp:790-810) */
  if (ex && n < CAP) { z[n] = 0; nz[n] = 0; type[n] |= T_SSA; n++; }
  if (im && n < CAP) { z[n] = 0; nz[n] = 0; type[n] |= T_NVA; n++; }
  *vo = (al > bes) ? (al - bes) : 0;
  *vss = P->explicit_ss ? (ssb - ssa) : (-al + bes + tc - nvb + nva);
  *tc_out = tc;
  return n;
}

typedef struct {
  float VoF, VssF;             /* Pairing float accumulators (STomoSh_INT3.cpp:375-392) */
  int64_t Vo64, Vss64, Vtc64;  /* exact totals */
  int64_t entries, columns;
  int n_bed;
} orient_t;

/* Per-column values are kept so that dumps can read them. */
typedef struct { int32_t* vo; int32_t* vss; int32_t* tc; } colvals_t;

/* Pairing (STomoSh_INT3.cpp:366-395): dirty slots ascending, columns with
 * more than one pixel. */
static void pairing(ws_t* w, const params_t* P, orient_t* o, const colvals_t* cv)
{
  qsort(w->dirty, (size_t)w->n_dirty, sizeof(int32_t), cmp_i32);
  const float thr = tomo_oracle_threshold(P->theta_c);
  float vof = 0.f, vssf = 0.f;
  int64_t vo64 = 0, vss64 = 0, tc64 = 0, ent = 0;
  for (int i = 0; i < w->n_dirty; i++) {
    const int32_t s = w->dirty[i];
    const size_t base = (size_t)s * ROWS;
    const int n = w->cnt[s];
    ent += n;
    int32_t vo = 0, vss = 0, tc = 0;
    if (n > 1) {
      w->cnt[s] = (uint8_t)pair_column(w->z + base, w->nz + base, w->type + base, n, P, thr, &vo, &vss, &tc);
      vof += (float)vo;
      vssf += (float)vss;
    }
    vo64 += vo; vss64 += vss; tc64 += tc;
    if (cv) { cv->vo[s] = vo; cv->vss[s] = vss; cv->tc[s] = tc; }
  }
  o->VoF = vof; o->VssF = vssf;
  o->Vo64 = vo64; o->Vss64 = vss64; o->Vtc64 = tc64;
  o->entries = ent; o->columns = w->n_dirty;
}

/* IsBedCandidate (STomoSh_INT3.cpp:1331-1373) */
static int bed_candidate(const ws_t* w, const params_t* P, int X, int Y)
{
  const int g = w->g;
  const int radius = (int)P->bed_outer;
  float min_dist = 1e5f;
  const int xa = (X - radius > 0) ? X - radius : 0, xb = (X + radius < g) ? X + radius : g;
  const int ya = (Y - radius > 0) ? Y - radius : 0, yb = (Y + radius < g) ? Y + radius : g;
  for (int sx = xa; sx < xb; sx++)
    for (int sy = ya; sy < yb; sy++) {
      const int32_t s = sx * g + sy;
      const int n = w->cnt[s];
      if (n > 0) {
        const size_t r = (size_t)s * ROWS + (size_t)(n - 1);
        const float dxf = (float)X - (float)sx, dyf = (float)Y - (float)sy;
        const float dist = sqrtf(dxf * dxf + dyf * dyf);
        const int t = w->type[r];
        if (w->z[r] == 0 && ((t & T_AL) || (t & T_BE) || (t & T_SSA) || (t & T_SS)))
          min_dist = (min_dist < dist) ? min_dist : dist;
      }
    }
  if (min_dist > P->bed_outer) return 0;
  if (P->bed_type == BED_BRIM || P->bed_type == BED_RAFT) return 1;
  if (P->bed_type == BED_SKIRT && min_dist > P->bed_inner) return 1;
  return 0;
}

/* GenerateBed (STomoSh_INT3.cpp:1375-1443) */
static void generate_bed(ws_t* w, const params_t* P, orient_t* o)
{
  o->n_bed = 0;
  if (P->bed_type == BED_NONE) return;
  if (w->n_dirty == 0) return;
  const int g = w->g;
  int minX = g, minY = g, maxX = -1, maxY = -1;
  for (int i = 0; i < w->n_dirty; i++) {
    const int sx = w->dirty[i] / g, sy = w->dirty[i] % g;
    if (sx < minX) minX = sx;
    if (sx > maxX) maxX = sx;
    if (sy < minY) minY = sy;
    if (sy > maxY) maxY = sy;
  }
  const int m = (int)P->bed_outer + 1;
  const int bx0 = (minX - m > 0) ? minX - m : 0, bx1 = (maxX + m + 1 < g) ? maxX + m + 1 : g;
  const int by0 = (minY - m > 0) ? minY - m : 0, by1 = (maxY + m + 1 < g) ? maxY + m + 1 : g;
  /* The scan reads the live slot state, as the reference does: a raft pixel
   * appended under a floor-level beta/SSA pixel becomes that slot's last
   * pixel (z = 1), so the slot stops counting as floor contact for slots
   * scanned after it. */
  for (int X = bx0; X < bx1; X++)
    for (int Y = by0; Y < by1; Y++) {
      const int32_t s = X * g + Y;
      const int n = w->cnt[s];
      int possible = 0;
      if (n == 0) possible = 1;
      else {
        const size_t r = (size_t)s * ROWS + (size_t)(n - 1);
        const int t = w->type[r];
        if (w->z[r] == 0) {
          if (t == T_NVA || t == T_VO || t == T_VSS) possible = 1;
          if ((t & T_AL) || (t & T_BE) || (t & T_SSA) || (t & T_SS)) possible = 0;
          if (P->bed_type == BED_RAFT && ((t & T_BE) || (t & T_SSA))) possible = 1;
        }
      }
      if (possible && bed_candidate(w, P, X, Y)) {
        const float pxl[3] = {(float)X, (float)Y, 1.f};
        const float nrm[3] = {0.f, 0.f, 0.f};
        set_bit(w, pxl, nrm, T_BED);
      }
    }
}

/* Calculate (STomoSh_INT3.cpp:1211-1255): float folds over dirty slots in
 * ascending order, then VolToMass. */
static void calculate(ws_t* w, const params_t* P, const orient_t* o, float vm[22],
                      const float* f32info, const int32_t* i32info)
{
  memset(vm, 0, 22 * sizeof(float));
  vm[8] = o->VoF;
  vm[4] = o->VssF;
  qsort(w->dirty, (size_t)w->n_dirty, sizeof(int32_t), cmp_i32);
  for (int i = 0; i < w->n_dirty; i++) {
    const size_t base = (size_t)w->dirty[i] * ROWS;
    const int n = w->cnt[w->dirty[i]];
    int32_t sa = 0, sb = 0, snvb = 0, snva = 0, stc = 0, sbed = 0;
    for (int p = 0; p < n; p++) {
      const int t = w->type[base + p];
      const int32_t zz = w->z[base + p];
      if (t & T_AL) sa += zz;
      if (t & T_BE) sb += zz;
      if (t & T_NVB) snvb += zz;
      if (t & T_NVA) snva += zz;
      if (t & T_TC) stc += zz;
      if (t & T_BED) sbed += zz;
    }
    vm[0] += (float)sa;
    vm[1] += (float)sb;
    vm[3] += (float)(snvb - snva);
    vm[2] += (float)stc;
    vm[11] += (float)sbed * P->bed_thickness;
  }
  tomo_oracle_vol_to_mass(f32info, i32info, vm);
}

/* VolToMass (STomoVolMassInfo.cpp:42-80).  Field order of vm_info
 * (STomoVolMassInfo.h:19-33): Va Vb Vtc Vnv | Vss Vss_clad Vss_core Ass_clad |
 * Vo Vo_clad Vo_core | Vbed Mbed | Mss Mss_clad Mss_core | Mo Mo_clad Mo_core |
 * Mtotal SS_vol */
void tomo_oracle_vol_to_mass(const float* f32info, const int32_t* i32info, float* vm)
{
  params_t P;
  read_params(f32info, i32info, &P);
  float Vss = vm[4], Vo = vm[8], Vbed = vm[11];
  float Vo_clad, Vo_core, Mo_clad, Mo_core, Mo;
  float Vss_clad = 0.f, Vss_core = 0.f, Ass_clad = 0.f, Mss_clad = 0.f, Mss_core = 0.f, Mss = 0.f;
  Vo_clad = P.surface_area * P.wall;
  Vo_core = Vo - Vo_clad;
  Mo_clad = Vo_clad * P.Fclad * P.rho;
  Mo_core = Vo_core * P.Fcore * P.rho;
  Mo = Mo_core + Mo_clad;
  if (P.explicit_ss) {
    if (Vss > MARGIN) {
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

/* ---- orientation driver ---- */
static int run_orientation(ws_t* w, const params_t* P, const float* f32info, const int32_t* i32info,
                           const float* ypr, int id, const int32_t* tri, const float* vtx, const float* vnrm,
                           orient_t* o, float vm[22], float mat16[16], const colvals_t* cv)
{
  rotate(w, P, vtx, vnrm, ypr[id * 3 + 0], ypr[id * 3 + 1], ypr[id * 3 + 2], mat16);
  pixelize(w, P, tri);
  if (w->error) return w->error;
  pairing(w, P, o, cv);
  generate_bed(w, P, o);
  if (w->error) return w->error;
  calculate(w, P, o, vm, f32info, i32info);
  return 0;
}

typedef struct {
  const float* f32info; const int32_t* i32info; const float* ypr;
  const int32_t* tri; const float* vtx; const float* vnrm;
  const params_t* P;
  int grid;
  float *Mo, *Mss, *Vtc, *VoF, *VssF;
  int64_t *Vo64, *Vss64, *Vtc64, *n_entries, *n_columns;
  int next;
  int error;
  pthread_mutex_t lock;
} sweep_t;

static void* sweep_worker(void* arg)
{
  sweep_t* S = (sweep_t*)arg;
  ws_t w;
  if (ws_init(&w, S->grid, S->P->n_vtx) != 0) {
    pthread_mutex_lock(&S->lock); S->error = -2; pthread_mutex_unlock(&S->lock);
    ws_free(&w);
    return NULL;
  }
  for (;;) {
    pthread_mutex_lock(&S->lock);
    const int id = (S->error == 0) ? S->next++ : S->P->n_ypr;
    pthread_mutex_unlock(&S->lock);
    if (id >= S->P->n_ypr) break;
    orient_t o;
    float vm[22];
    memset(&o, 0, sizeof(o));
    const int rc = run_orientation(&w, S->P, S->f32info, S->i32info, S->ypr, id, S->tri, S->vtx, S->vnrm,
                                   &o, vm, NULL, NULL);
    if (rc != 0) {
      pthread_mutex_lock(&S->lock); S->error = rc; pthread_mutex_unlock(&S->lock);
      break;
    }
    if (S->Mo) S->Mo[id] = vm[16];
    if (S->Mss) S->Mss[id] = vm[13];
    if (S->Vtc) S->Vtc[id] = vm[2];
    if (S->VoF) S->VoF[id] = o.VoF;
    if (S->VssF) S->VssF[id] = o.VssF;
    if (S->Vo64) S->Vo64[id] = o.Vo64;
    if (S->Vss64) S->Vss64[id] = o.Vss64;
    if (S->Vtc64) S->Vtc64[id] = o.Vtc64;
    if (S->n_entries) S->n_entries[id] = o.entries;
    if (S->n_columns) S->n_columns[id] = o.columns;
  }
  ws_free(&w);
  return NULL;
}

/* _find1stOptimal (Tomo_Shell2026.cpp:89-97) */
static int first_optimal(int n, const float* mss)
{
  if (n <= 1) return 0;
  int idx = 0;
  float best = 1e5f;
  for (int i = 0; i < n; i++)
    if (mss[i] < best) { best = mss[i]; idx = i; }
  return idx;
}

int tomo_oracle_sweep(const float* f32info, const int32_t* i32info, const float* ypr,
                      const int32_t* tri, const float* vtx, const float* vnrm,
                      int grid, int n_threads,
                      float* Mo, float* Mss, float* Vtc, float* VoF, float* VssF,
                      int64_t* Vo64, int64_t* Vss64, int64_t* Vtc64,
                      int64_t* n_entries, int64_t* n_columns)
{
  if (!f32info || !i32info || !ypr || !tri || !vtx || !vnrm) return -1;
  params_t P;
  read_params(f32info, i32info, &P);
  if (P.n_ypr < 0 || P.n_tri < 0 || P.n_vtx < 0) return -1;
  float* mss_local = NULL;
  if (!Mss) {
    mss_local = malloc(sizeof(float) * (size_t)(P.n_ypr > 0 ? P.n_ypr : 1));
    if (!mss_local) return -2;
    Mss = mss_local;
  }
  sweep_t S;
  memset(&S, 0, sizeof(S));
  S.f32info = f32info; S.i32info = i32info; S.ypr = ypr; S.tri = tri; S.vtx = vtx; S.vnrm = vnrm;
  S.P = &P; S.grid = grid > 0 ? grid : 256;
  S.Mo = Mo; S.Mss = Mss; S.Vtc = Vtc; S.VoF = VoF; S.VssF = VssF;
  S.Vo64 = Vo64; S.Vss64 = Vss64; S.Vtc64 = Vtc64; S.n_entries = n_entries; S.n_columns = n_columns;
  pthread_mutex_init(&S.lock, NULL);
  int nt = n_threads < 1 ? 1 : n_threads;
  if (nt > P.n_ypr) nt = P.n_ypr > 0 ? P.n_ypr : 1;
  pthread_t* th = malloc(sizeof(pthread_t) * (size_t)nt);
  if (!th) { free(mss_local); return -2; }
  for (int i = 0; i < nt; i++) pthread_create(&th[i], NULL, sweep_worker, &S);
  for (int i = 0; i < nt; i++) pthread_join(th[i], NULL);
  free(th);
  pthread_mutex_destroy(&S.lock);
  const int rc = (S.error != 0) ? S.error : first_optimal(P.n_ypr, Mss);
  free(mss_local);
  return rc;
}

int tomo_oracle_columns(const float* f32info, const int32_t* i32info, const float* ypr,
                        const int32_t* tri, const float* vtx, const float* vnrm,
                        int ypr_index, int grid,
                        int32_t* n_vox, int16_t* vox_zn, int32_t* n_fin, int16_t* fin_tzn,
                        int32_t* col_vo, int32_t* col_vss, int32_t* col_vtc,
                        float* vm22, float* mat16)
{
  if (!f32info || !i32info || !ypr || !tri || !vtx || !vnrm) return -1;
  params_t P;
  read_params(f32info, i32info, &P);
  if (ypr_index < 0 || ypr_index >= P.n_ypr) return -1;
  const int g = grid > 0 ? grid : 256;
  const size_t ns = (size_t)g * g;
  ws_t w;
  if (ws_init(&w, g, P.n_vtx) != 0) { ws_free(&w); return -2; }
  colvals_t cv;
  cv.vo = calloc(ns, sizeof(int32_t));
  cv.vss = calloc(ns, sizeof(int32_t));
  cv.tc = calloc(ns, sizeof(int32_t));
  if (!cv.vo || !cv.vss || !cv.tc) { ws_free(&w); free(cv.vo); free(cv.vss); free(cv.tc); return -2; }
  orient_t o;
  memset(&o, 0, sizeof(o));
  float vm[22], mat[16];
  rotate(&w, &P, vtx, vnrm, ypr[ypr_index * 3 + 0], ypr[ypr_index * 3 + 1], ypr[ypr_index * 3 + 2], mat);
  pixelize(&w, &P, tri);
  int rc = w.error;
  if (rc == 0) {
    for (size_t s = 0; s < ns; s++) {
      if (n_vox) n_vox[s] = w.cnt[s];
      if (vox_zn)
        for (int p = 0; p < ROWS; p++) {
          vox_zn[(s * ROWS + (size_t)p) * 2 + 0] = w.z[s * ROWS + (size_t)p];
          vox_zn[(s * ROWS + (size_t)p) * 2 + 1] = w.nz[s * ROWS + (size_t)p];
        }
    }
    pairing(&w, &P, &o, &cv);
    generate_bed(&w, &P, &o);
    rc = w.error;
  }
  if (rc == 0) {
    calculate(&w, &P, &o, vm, f32info, i32info);
    for (size_t s = 0; s < ns; s++) {
      if (n_fin) n_fin[s] = w.cnt[s];
      if (fin_tzn)
        for (int p = 0; p < ROWS; p++) {
          fin_tzn[(s * ROWS + (size_t)p) * 3 + 0] = w.type[s * ROWS + (size_t)p];
          fin_tzn[(s * ROWS + (size_t)p) * 3 + 1] = w.z[s * ROWS + (size_t)p];
          fin_tzn[(s * ROWS + (size_t)p) * 3 + 2] = w.nz[s * ROWS + (size_t)p];
        }
      if (col_vo) col_vo[s] = cv.vo[s];
      if (col_vss) col_vss[s] = cv.vss[s];
      if (col_vtc) col_vtc[s] = cv.tc[s];
    }
    if (vm22) memcpy(vm22, vm, sizeof(vm));
    if (mat16) memcpy(mat16, mat, sizeof(mat));
  }
  ws_free(&w);
  free(cv.vo); free(cv.vss); free(cv.tc);
  return rc;
}
