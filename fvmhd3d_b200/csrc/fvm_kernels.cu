// sm_100a kernels of the fvmhd3d fluid hot path and the C-ABI context
// (include/fvmhd3d_b200.h).
//
// Data layout in HBM (one record per cell / face, 16-byte aligned):
//   faces  s12 int2, geo double4 (unit normal, area), cen double4 (centroid)
//   cells  U double[10], dU double[14], Wrec double[50] (w,x,y,z,t),
//          pos/vel double[3], tlast/tend/volp double, rung/bnd int,
//          CSR off[n+1] / lnk[] of face ids (cell face order of the mesh)
//
// Stage kernels follow the reference call sequence (MPI/iterate.cpp:95-113).
// Per-cell reductions over faces (limiter min/max, tau, gradients, timestep,
// flux sums) are gathers in the cell's face order, so every run gives the
// same bits.  Each face flux is evaluated once by a face-parallel kernel that
// stores the face's contribution; the owning cells then gather it.
#include "fvm_math.cuh"
#include "flux_mlp.cuh"
#include "mlp_train.cuh"
#include "flux_learn.cuh"
#include "../../include/fvmhd3d_b200.h"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <string>
#include <algorithm>

using namespace fvm;

// Minimum resident 128-thread blocks per SM for the face-flux kernels (caps
// their registers: 3 -> 168 for FP64, 4 -> 128 for FP32, no spills).
#ifndef FVM_FLUX_MINB_D
#define FVM_FLUX_MINB_D 3
#endif
#ifndef FVM_FLUX_MINB_F
#define FVM_FLUX_MINB_F 4
#endif
#define FVM_FLUX_MINB(R) (sizeof(R) == 4 ? FVM_FLUX_MINB_F : FVM_FLUX_MINB_D)
#ifndef FVM_CELL_LFJ
#define FVM_CELL_LFJ 1  // cell kernels take (face, neighbour) from the link table instead of s12
#endif
#ifndef FVM_CELL_UNROLL
#define FVM_CELL_UNROLL 1  // unroll factor of the cell kernels' face loops (1 and 2 time the same within 1%)
#endif
#ifndef FVM_REUSE_MINMAX
#define FVM_REUSE_MINMAX 1  // the limiter reuses the reconstruction's neighbour min/max when every cell steps
#endif
#define FVM_PRAGMA(x) _Pragma(#x)
#define FVM_CELL_LOOP_(n) FVM_PRAGMA(unroll n)
#define FVM_CELL_LOOP FVM_CELL_LOOP_(FVM_CELL_UNROLL)
#ifndef FVM_LIMITER_STAGE
#define FVM_LIMITER_STAGE 1  // default: limiter face records staged in shared memory per block
#endif
#ifndef FVM_ADJUST_REPLAY
#define FVM_ADJUST_REPLAY 1  // adjust_timesteps by parallel replay (sequential sweep as fallback)
#endif
// Thread-to-cell indirection: inside each window of CPW consecutive cells the
// threads visit cells in order of face count, so the lanes of a warp run face
// loops of similar length (less divergence) while memory locality stays
// within the window.  Pure relabelling of which thread does which cell.
#ifndef FVM_CELL_PERM
#define FVM_CELL_PERM 0
#endif
constexpr int CPW = 64;

namespace {

enum : unsigned char { A_ACTIVE = 1, A_LNGB = 2, A_HASNGB = 4 };
enum : unsigned char { F_SWAP = 1, F_SKIPJ = 2, F_OFF = 4 };

// Scheduler state kept on the device so that a whole step is a fixed
// sequence of launches (MPI/Scheduler.h:4-30, 108-154).
struct Sched {
  unsigned long long tsysU, flags;
  double t_global, dtmin;
  int min_rung, max_rung;
  int iscal[8];  // [0] rung maximum, [1] active cells, [2] error flags, [3] active faces,
                 // [4] dirty sites of adjust_timesteps, [5] active non-boundary sites,
                 // [6] adjust_timesteps replays, [7] 1 if the sequential sweep ran
  unsigned long long nactive_total, nfaces_total, steps;
  unsigned long long tprevU;  // tsysU before the last pull_active_list
  int mnmx_ok;                // the last step reconstructed every cell (its min/max are current)
  double sink;                // written only by a calibration kernel, never in practice
  int ninv;                   // cells in the involved-cell list of a partial step
};

struct Dev {
  // mesh
  int2 *s12;
  double4 *geo, *cen, *dr1, *dr2;
  double *cvol, *ccen;
  int *off, *lnk;
  int *perm;  // thread slot -> cell (face-count order inside windows of CPW cells)
  int *alist, *bcount;  // ordered active-site list and block offsets (individual timesteps)
  int *flist, *fbcount; // ordered active-face list and its block offsets (partial steps)
  int *clist, *cbcount; // ordered list of the step's active and neighbour cells, block offsets (partial steps)
  unsigned char *bnb;   // per cell: 1 when a neighbour is a boundary cell (set with the boundary codes)
  int2 *lfj;            // per link: face id, neighbour (~j when the cell is s2)
  int *lsort, *lpart;   // per link: links of the cell by ascending neighbour; the same face's other link
  double *rdv, *wrv, *dt0;  // adjust_timesteps replay state (per link, per link, per cell)
  int *aflag;               // adjust_timesteps replay flags
  unsigned char *awork;     // adjust_timesteps replay work lists (2 per cell)
  void *mnmx;               // per cell: the reconstruction's neighbour min and max (20 of the bulk type)
  void *lrw;                // per link: the reconstruction's face weights (6, bulk type)
  void *lrd;                // per link: the face centroid's offset from the cell (3, bulk type)
  void *lld;                // per link: the limiter's face-side offset dr (3, bulk type)
  unsigned char *mz;        // per cell: the reconstruction met a boundary (the limiter is zero)
  // learned-flux buffers (fvm_set_flux_mode)
  void *lX, *lY, *lface, *lcount, *lstats, *lhx, *lhy, *lhcount, *lnorm;
  // state
  double *pos, *vel, *tlast, *tend, *volp;
  double *opos, *ovel;  // orig_pos / orig_vel of correct() (generator motion)
  float *divb;          // divBi of collect_results (float, as the reference keeps it)
  int *rung, *bnd;
  double *U, *dU;
  void *Wrec;  // bulk type (double or float), ncell x 50
  // per-step work
  unsigned char *act0, *act, *hash, *fcode, *fcode2, *fflag;
  void *tau, *fcon, *fcon2, *Wst, *fst;  // bulk type
  double *dtl, *stepdU;
  Sched *S;
  unsigned long long *counters;
};

__device__ __forceinline__ bool face_active(const unsigned char *act, const int *bnd, int a, int b) {
  return ((act[a] & A_ACTIVE) && bnd[a] == NO_BOUNDARY) || ((act[b] & A_ACTIVE) && bnd[b] == NO_BOUNDARY);
}

__device__ __forceinline__ void ld3(const double *p, double *o) { o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; }

// ---- begin_step: active flags (Scheduler::pull_active_list) ---------------
__global__ void k_active(int n, const int *__restrict__ rung, const Sched *__restrict__ S,
                         unsigned char *__restrict__ act, int *__restrict__ nactive) {
  const unsigned long long flags = S->flags;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool a = false;
  if (i < n) {
    const int r = rung[i];
    a = r >= 0 && r < RUNGMAX && ((flags >> (RUNGMAX - 1 - r)) & 1ULL);
    act[i] = a ? A_ACTIVE : 0;
  }
  __shared__ int bsum;
  if (threadIdx.x == 0) bsum = 0;
  __syncthreads();
  const unsigned cnt = __popc(__ballot_sync(0xffffffffu, a));
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&bsum, (int)cnt);
  __syncthreads();
  if (threadIdx.x == 0 && bsum) atomicAdd(nactive, bsum);
}

// per-step face flags: active face (a face of an active non-boundary cell,
// MPI/iterate.cpp:58-93) and the boundary flags of its two cells
enum : unsigned char { FF_ACTIVE = 1, FF_BND1 = 2, FF_BND2 = 4 };
// Per face: active flag and boundary flags, and the site flags of
// build_mesh_active (MPI/build_mesh_active.cpp:524-528): a face between an
// active and an inactive cell marks the inactive one a local neighbour and the
// active one as having one.  A cell only ever receives one kind of mark, so
// concurrent byte stores to it write the same value; the active bit they
// test never changes during this kernel.
__global__ void k_faceflags(int nf, const int2 *__restrict__ s12, unsigned char *__restrict__ act,
                            const int *__restrict__ bnd, unsigned char *__restrict__ fflag,
                            int *__restrict__ nface_active, unsigned char *__restrict__ fcode,
                            unsigned char *__restrict__ fcode2, int *__restrict__ bcount) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  bool a = false;
  if (f < nf) {
    const int2 e = s12[f];
    const bool a1 = act[e.x] & A_ACTIVE, a2 = act[e.y] & A_ACTIVE;
    const bool b1 = bnd[e.x] != NO_BOUNDARY, b2 = bnd[e.y] != NO_BOUNDARY;
    a = (a1 && !b1) || (a2 && !b2);
    unsigned char v = a ? FF_ACTIVE : 0;
    if (b1) v |= FF_BND1;
    if (b2) v |= FF_BND2;
    const unsigned char was = fflag[f];
    fflag[f] = v;
    // the flux passes visit active faces only: a face that goes inactive is
    // coded F_OFF (codes start F_OFF when the state is installed)
    if (!a && (was & FF_ACTIVE)) { fcode[f] = F_OFF; fcode2[f] = F_OFF; }
    if (a1 != a2) {
      act[a1 ? e.y : e.x] = A_LNGB;
      act[a1 ? e.x : e.y] = A_ACTIVE | A_HASNGB;
    }
  }
  __shared__ int bsum;
  if (threadIdx.x == 0) bsum = 0;
  __syncthreads();
  const unsigned cnt = __popc(__ballot_sync(0xffffffffu, a));
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&bsum, (int)cnt);
  __syncthreads();
  if (threadIdx.x == 0 && bsum) atomicAdd(nface_active, bsum);
  if (bcount && threadIdx.x == 0) bcount[blockIdx.x] = bsum;  // per-block counts of the face compaction
}

// Face offsets used by every face loop, computed once per generator layout:
//   dr1 = centroid - x_s1 (the reference's dri, MPI/compute_update.cpp:136)
//         with w = dri . n (dsh, :164)
//   dr2 = wrap(centroid - x_s2) (MPI/compute_reconstruction.cpp:74-83 seen
//         from s2)
__global__ void k_face_geom(int nf, Params P, const int2 *__restrict__ s12, const double4 *__restrict__ geo,
                            const double4 *__restrict__ cen, const double *__restrict__ pos,
                            double4 *__restrict__ dr1, double4 *__restrict__ dr2) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int2 e = s12[f];
  const double4 g = geo[f], c = cen[f];
  const double *pa = pos + 3 * (size_t)e.x, *pb = pos + 3 * (size_t)e.y;
  const double d1[3] = {c.x - pa[0], c.y - pa[1], c.z - pa[2]};
  double d2[3] = {c.x - pb[0], c.y - pb[1], c.z - pb[2]};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double L = P.box[a];
    if (d2[a] > 0.5 * L) d2[a] -= L;
    else if (d2[a] < -0.5 * L) d2[a] += L;
  }
  dr1[f] = make_double4(d1[0], d1[1], d1[2], d1[0] * g.x + d1[1] * g.y + d1[2] * g.z);
  dr2[f] = make_double4(d2[0], d2[1], d2[2], 0.0);
}

// min-image of the s1 offset for the reconstruction (a no-op for meshes that
// keep the centroid in the frame of s1, as the reference asserts)
__device__ __forceinline__ void wrap3(const Params &P, double *d) {
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double L = P.box[a];
    if (d[a] > 0.5 * L) d[a] -= L;
    else if (d[a] < -0.5 * L) d[a] += L;
  }
}

// Geometry of one face side for the reconstruction
// (MPI/compute_reconstruction.cpp:70-138): the min-image offset d of the face
// centroid, the normal oriented along it and the normal distance dsh.
__device__ __forceinline__ void recon_geom(const Params &P, bool own, const double4 &g, const double4 &o4, double *d,
                                           double *nrm, double &dsh) {
  d[0] = o4.x; d[1] = o4.y; d[2] = o4.z;
  if (own) wrap3(P, d);
  const double sgn = (d[0] * g.x + d[1] * g.y + d[2] * g.z) < 0.0 ? -1.0 : 1.0;
  nrm[0] = g.x * sgn; nrm[1] = g.y * sgn; nrm[2] = g.z * sgn;
  dsh = d[0] * nrm[0] + d[1] * nrm[1] + d[2] * nrm[2];
}
// A / (2 dsh), the face weight of the gradient.
__device__ __forceinline__ double recon_ia(const double4 &g, double dsh) {
  return g.w * ((dsh != 0.0) ? 0.5 / dsh : 0.0);
}

// The reconstruction's per-link records, computed once per mesh (the mesh is
// fixed while it is installed).  The face term of the gradient,
// ((wj + wi) dsh n + (wj - wi) (d - dsh n)) A / (2 dsh), becomes
// (wj + wi) a + (wj - wi) b with a = dsh n A/(2 dsh), b = (d - dsh n) A/(2 dsh)
// (lrw: a then b), and the limiter pass reads the min-image offset d (lrd).
// The face loops then do no geometry, no division and one dependent load.
template <typename R>
__global__ void k_link_recon(int n, Params P, const int *__restrict__ off, const int2 *__restrict__ lfj,
                             const double4 *__restrict__ geo, const double4 *__restrict__ dr1,
                             const double4 *__restrict__ dr2, R *__restrict__ lrw, R *__restrict__ lrd,
                             R *__restrict__ lld) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int2 fj = lfj[q];
    const bool own = fj.y >= 0;
    const double4 g = geo[fj.x];
    double d[3], nrm[3], dsh;
    recon_geom(P, own, g, own ? dr1[fj.x] : dr2[fj.x], d, nrm, dsh);
    const double ia = recon_ia(g, dsh);
    R *w = lrw + 6 * (size_t)q, *o = lrd + 3 * (size_t)q;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      w[a] = R(nrm[a] * dsh * ia);
      w[3 + a] = R((d[a] - nrm[a] * dsh) * ia);
      o[a] = R(d[a]);
    }
    // the limiter's offset of this side: dri for s1, dri - 2 dsh n for s2
    // (MPI/compute_update.cpp:157-212; dr1 unwrapped, as the limiter uses it)
    const double4 e = dr1[fj.x];
    const double dsl = own ? 0.0 : 2.0 * e.w;
    R *l3 = lld + 3 * (size_t)q;
    l3[0] = R(e.x - g.x * dsl); l3[1] = R(e.y - g.y * dsl); l3[2] = R(e.z - g.z * dsl);
  }
}

// ---- slope_limiter (MPI/compute_reconstruction.cpp:201-602) --------------
// TPC threads per imported cell, each owning KH of the ten primitives: face
// pass 1 (min/max of neighbour differences) and face pass 2 (limiter of the
// space+time extrapolated difference) over the cell's active faces.  The
// result tau is applied on the fly by the corrector, so Wrec is not modified.
// R is the bulk type (double: plain path; float: FP32 path); face geometry
// stays double and is rounded to R only where it multiplies bulk data.
// KH primitives per thread, TPC = 10 / KH threads per cell, and the blocks
// per SM that the launch bounds ask for, per bulk type.  Timed on B200 on the
// 128^3 blast: two primitives per thread (five threads per cell) give the
// limiter and the FP64 reconstruction the occupancy that hides their loads;
// the FP32 reconstruction is faster with five per thread.
template <typename R> struct CellTune;
template <> struct CellTune<double> {
#ifndef FVM_RECON_MINB_D
#define FVM_RECON_MINB_D 8
#endif
  static constexpr int KH_LIM = 2, MINB_LIM = 6, KH_REC = 2, MINB_REC = FVM_RECON_MINB_D;
};
template <> struct CellTune<float> {
  static constexpr int KH_LIM = 2, MINB_LIM = 8, KH_REC = 5, MINB_REC = 6;
};

// KH consecutive bulk values from p, as 2-wide loads when KH is even: the
// callers' rows (10 or 50 values per cell, 6 per link) and even offsets then
// start on 16-byte (FP64) or 8-byte (FP32) boundaries.
template <typename R> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float2; };
template <typename R, int N>
__device__ __forceinline__ void load_n(const R *__restrict__ p, R *v) {
  if constexpr (N % 2 == 0) {
    using V = typename Vec2<R>::T;
    const V *p2 = reinterpret_cast<const V *>(p);
#pragma unroll
    for (int h = 0; h < N / 2; h++) { const V x = p2[h]; v[2 * h] = x.x; v[2 * h + 1] = x.y; }
  } else {
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = p[k];
  }
}

template <typename R, int N>
__device__ __forceinline__ void store_n(R *__restrict__ p, const R *v) {
  if constexpr (N % 2 == 0) {
    using V = typename Vec2<R>::T;
    V *p2 = reinterpret_cast<V *>(p);
#pragma unroll
    for (int h = 0; h < N / 2; h++) { V x; x.x = v[2 * h]; x.y = v[2 * h + 1]; p2[h] = x; }
  } else {
#pragma unroll
    for (int k = 0; k < N; k++) p[k] = v[k];
  }
}

// A face's 14 contributions as seven 2-wide stores (records of 112 bytes in
// FP64, 56 in FP32).
template <typename R>
__device__ __forceinline__ void store_contrib(R *__restrict__ o, const R *v) {
  using V = typename Vec2<R>::T;
  V *o2 = reinterpret_cast<V *>(o);
#pragma unroll
  for (int h = 0; h < 7; h++) { V x; x.x = v[2 * h]; x.y = v[2 * h + 1]; o2[h] = x; }
}

template <typename R, int KH>
__device__ __forceinline__ void limiter_thread(int i, int k0, bool reuse, double t_global,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ lfj, const int2 *__restrict__ s12,
    const double4 *__restrict__ geo, const double4 *__restrict__ dr1, const unsigned char *__restrict__ fflag,
    const unsigned char *__restrict__ act, const double *__restrict__ tlast,
    const R *__restrict__ Wrec, R *__restrict__ tau, R *__restrict__ fst,
    const R *__restrict__ mnmx, const unsigned char *__restrict__ mz, const R *__restrict__ lld) {
  if (!(act[i] & (A_ACTIVE | A_LNGB))) return;
  const double ti = tlast[i];
  const R *ri = Wrec + 50 * (size_t)i + k0;
  R mn[KH], mx[KH], ln[KH], lq[KH], wi[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { mn[k] = R(0); mx[k] = R(0); ln[k] = R(2); lq[k] = R(1); wi[k] = ri[k]; }
  const int q0 = off[i], q1 = off[i + 1];
  bool zero = false;
  if (reuse) {
    const R *mm = mnmx + 20 * (size_t)i + k0;
#pragma unroll
    for (int k = 0; k < KH; k++) { mn[k] = mm[k]; mx[k] = mm[10 + k]; }
    zero = mz[i] != 0;
  }
  // pass 1: min/max of neighbour differences over active interior faces
  FVM_CELL_LOOP
  for (int q = q0; q < (reuse ? q0 : q1); q++) {
#if FVM_CELL_LFJ
    const int2 fj = lfj[q];
    const int f = fj.x, j = fj.y >= 0 ? fj.y : ~fj.y;
    const unsigned char ff = fflag[f];
    if (!(ff & FF_ACTIVE)) continue;
    if (ff & (FF_BND1 | FF_BND2)) { zero = true; continue; }
#else
    const int f = lnk[q];
    const unsigned char ff = fflag[f];
    if (!(ff & FF_ACTIVE)) continue;
    if (ff & (FF_BND1 | FF_BND2)) { zero = true; continue; }
    const int2 e = s12[f];
    const int j = e.x == i ? e.y : e.x;
#endif
    R rj[KH];
    load_n<R, KH>(Wrec + 50 * (size_t)j + k0, rj);
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R diff = rj[k] - wi[k];
      mn[k] = smin(mn[k], diff);
      mx[k] = smax(mx[k], diff);
    }
  }
  R *to = tau + 10 * (size_t)i + k0;
  R gx[KH], gy[KH], gz[KH], gt[KH];
  if (zero) {
    // a boundary face zeroes the limiter: the face states are w itself
#pragma unroll
    for (int k = 0; k < KH; k++) { to[k] = R(0); gx[k] = gy[k] = gz[k] = gt[k] = R(0); }
  } else {
    R thr[KH];
#pragma unroll
    for (int k = 0; k < KH; k++) {
      gx[k] = ri[10 + k]; gy[k] = ri[20 + k]; gz[k] = ri[30 + k]; gt[k] = ri[40 + k];
      thr[k] = limiter_thr(mn[k], mx[k]);
    }
    // pass 2: limiter of the extrapolated difference at each active face
    FVM_CELL_LOOP
    for (int q = q0; q < q1; q++) {
#if FVM_CELL_LFJ
      const int2 fj = lfj[q];
      const int f = fj.x;
      if (!(fflag[f] & FF_ACTIVE)) continue;
      const bool own = fj.y >= 0;
      const double tj = tlast[own ? fj.y : ~fj.y];
      const double dtI = t_global - (own ? ti : tj), dtJ = t_global - (own ? tj : ti);
#else
      const int f = lnk[q];
      if (!(fflag[f] & FF_ACTIVE)) continue;
      const int2 e = s12[f];
      const double dtI = t_global - tlast[e.x], dtJ = t_global - tlast[e.y];
      const bool own = e.x == i;
#endif
      const double dth = 0.5 * smin(dtI, dtJ);
      const R *l3 = lld + 3 * (size_t)q;
      const R dr[3] = {l3[0], l3[1], l3[2]};
      const R dtt = R(own ? dtI - dth : dtJ - dth);
#pragma unroll
      for (int k = 0; k < KH; k++) {
        const R dWx = gx[k] * dr[0] + gy[k] * dr[1] + gz[k] * dr[2];
        const R dW = dWx + gt[k] * dtt;
        limiter_ratio(ln[k], lq[k], dW, mn[k], mx[k], thr[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R tk = limiter_finish(ln[k], lq[k]);
      to[k] = tk;
      gx[k] *= tk; gy[k] *= tk; gz[k] *= tk; gt[k] *= tk;
    }
  }
  // pass 3: the half-step extrapolated state of this cell at each active
  // interior face (MPI/compute_update.cpp:157-212), stored per face side
  FVM_CELL_LOOP
  for (int q = q0; q < q1; q++) {
#if FVM_CELL_LFJ
    const int2 fj = lfj[q];
    const int f = fj.x;
    const unsigned char ff = fflag[f];
    if (!(ff & FF_ACTIVE) || (ff & (FF_BND1 | FF_BND2))) continue;
    const bool own = fj.y >= 0;
    const double tj = tlast[own ? fj.y : ~fj.y];
    const double dtI = t_global - (own ? ti : tj), dtJ = t_global - (own ? tj : ti);
#else
    const int f = lnk[q];
    const unsigned char ff = fflag[f];
    if (!(ff & FF_ACTIVE) || (ff & (FF_BND1 | FF_BND2))) continue;
    const int2 e = s12[f];
    const double dtI = t_global - tlast[e.x], dtJ = t_global - tlast[e.y];
    const bool own = e.x == i;
#endif
    const double dt = smin(dtI, dtJ);
    const R *l3 = lld + 3 * (size_t)q;
    const R dr[3] = {l3[0], l3[1], l3[2]};
    const R dtt = R(own ? dtI - 0.5 * dt : dtJ - 0.5 * dt);
    R o[KH];
#pragma unroll
    for (int k = 0; k < KH; k++) o[k] = wi[k] + ((gx[k] * dr[0] + gy[k] * dr[1] + gz[k] * dr[2]) + gt[k] * dtt);
    store_n<R, KH>(fst + 20 * (size_t)f + (own ? 0 : 10) + k0, o);
  }
}

// Staged limiter: a block's CST cells (TPC threads each) first compute the
// per-face records of passes 2 and 3 (the side's offset dr, the two time
// offsets, the face and its flags) for all their faces together, into shared
// memory, so the face loops read no global memory but the cell's own record.
// Used when the first pass is reused (every cell steps) and the block's faces
// fit (LCAP); otherwise the block runs limiter_thread.
template <int KH> __host__ __device__ constexpr int limiter_cst() { return 128 / (10 / KH); }  // cells per block
template <int KH> __host__ __device__ constexpr int limiter_lcap() { return 22 * limiter_cst<KH>(); }
template <typename R, int KH>
constexpr int limiter_stage_bytes() { return limiter_lcap<KH>() * (5 * (int)sizeof(R) + 4); }

// One block's CST cells (cell block cb); called by every thread of the block.
template <typename R, int KH>
__device__ __forceinline__ void limiter_st_block(int cb, int n, bool reuse, double t_global, int *soff,
    unsigned char *lsm,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ lfj, const int2 *__restrict__ s12,
    const double4 *__restrict__ geo, const double4 *__restrict__ dr1, const unsigned char *__restrict__ fflag,
    const unsigned char *__restrict__ act, const double *__restrict__ tlast,
    const R *__restrict__ Wrec, R *__restrict__ tau, R *__restrict__ fst, const int *__restrict__ perm,
    const R *__restrict__ mnmx, const unsigned char *__restrict__ mz, const R *__restrict__ lld) {
  constexpr int TPC = 10 / KH, CST = limiter_cst<KH>(), LCAP = limiter_lcap<KH>();
  const int tid = threadIdx.x;
  const int c0 = cb * CST;
  const int c1 = c0 + CST < n ? c0 + CST : n;
  const int L0 = off[c0], nL = off[c1] - L0;
  const bool staged = reuse && nL <= LCAP;  // uniform over the block
  R *sdx = reinterpret_cast<R *>(lsm), *sdy = sdx + LCAP, *sdz = sdy + LCAP, *st2 = sdz + LCAP, *st3 = st2 + LCAP;
  int *sfk = reinterpret_cast<int *>(st3 + LCAP);
  if (staged) {
    for (int k = tid; k <= c1 - c0; k += blockDim.x) soff[k] = off[c0 + k] - L0;
    __syncthreads();
    for (int l = tid; l < nL; l += blockDim.x) {
      int lo = 0, hi = c1 - c0;  // soff[lo] <= l < soff[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (soff[mid] <= l) lo = mid; else hi = mid;
      }
      const int2 fj = lfj[L0 + l];
      const int f = fj.x;
      const bool own = fj.y >= 0;
      const unsigned char ff = fflag[f];
      const double ti = tlast[c0 + lo], tj = tlast[own ? fj.y : ~fj.y];
      const double dtI = t_global - (own ? ti : tj), dtJ = t_global - (own ? tj : ti);
      const double dth = 0.5 * smin(dtI, dtJ);
      const double dt = smin(dtI, dtJ);
      const R *l3 = lld + 3 * (size_t)(L0 + l);
      sdx[l] = l3[0];
      sdy[l] = l3[1];
      sdz[l] = l3[2];
      st2[l] = R(own ? dtI - dth : dtJ - dth);
      st3[l] = R(own ? dtI - 0.5 * dt : dtJ - 0.5 * dt);
      sfk[l] = (f << 3) | ((ff & FF_ACTIVE) ? 1 : 0) | ((ff & (FF_BND1 | FF_BND2)) ? 2 : 0) | (own ? 4 : 0);
    }
  }
  __syncthreads();
  const int cl = tid / TPC, k0 = (tid % TPC) * KH;
  if (cl >= CST || c0 + cl >= n) return;
  if (!staged) {
    limiter_thread<R, KH>(perm[c0 + cl], k0, reuse, t_global, off, lnk, lfj, s12, geo, dr1, fflag, act, tlast, Wrec, tau,
                          fst, mnmx, mz, lld);
    return;
  }
  const int i = c0 + cl;  // the staged blocks assume the identity thread-to-cell map
  if (!(act[i] & (A_ACTIVE | A_LNGB))) return;
  const R *ri = Wrec + 50 * (size_t)i + k0;
  R mn[KH], mx[KH], ln[KH], lq[KH], wi[KH], gx[KH], gy[KH], gz[KH], gt[KH];
  const R *mm = mnmx + 20 * (size_t)i + k0;
#pragma unroll
  for (int k = 0; k < KH; k++) {
    mn[k] = mm[k]; mx[k] = mm[10 + k]; ln[k] = R(2); lq[k] = R(1); wi[k] = ri[k];
  }
  const bool zero = mz[i] != 0;
  const int q0 = soff[cl], q1 = soff[cl + 1];
  R *to = tau + 10 * (size_t)i + k0;
  if (zero) {
#pragma unroll
    for (int k = 0; k < KH; k++) { to[k] = R(0); gx[k] = gy[k] = gz[k] = gt[k] = R(0); }
  } else {
    R thr[KH];
#pragma unroll
    for (int k = 0; k < KH; k++) {
      gx[k] = ri[10 + k]; gy[k] = ri[20 + k]; gz[k] = ri[30 + k]; gt[k] = ri[40 + k];
      thr[k] = limiter_thr(mn[k], mx[k]);
    }
    for (int l = q0; l < q1; l++) {
      if (!(sfk[l] & 1)) continue;
      const R d0 = sdx[l], d1 = sdy[l], d2 = sdz[l], dtt = st2[l];
#pragma unroll
      for (int k = 0; k < KH; k++) {
        const R dWx = gx[k] * d0 + gy[k] * d1 + gz[k] * d2;
        const R dW = dWx + gt[k] * dtt;
        limiter_ratio(ln[k], lq[k], dW, mn[k], mx[k], thr[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R tk = limiter_finish(ln[k], lq[k]);
      to[k] = tk;
      gx[k] *= tk; gy[k] *= tk; gz[k] *= tk; gt[k] *= tk;
    }
  }
  for (int l = q0; l < q1; l++) {
    const int fk = sfk[l];
    if (!(fk & 1) || (fk & 2)) continue;
    const R d0 = sdx[l], d1 = sdy[l], d2 = sdz[l], dtt = st3[l];
    R o[KH];
#pragma unroll
    for (int k = 0; k < KH; k++) o[k] = wi[k] + ((gx[k] * d0 + gy[k] * d1 + gz[k] * d2) + gt[k] * dtt);
    store_n<R, KH>(fst + 20 * (size_t)(fk >> 3) + ((fk & 4) ? 0 : 10) + k0, o);
  }
}

// One block per CST cells; with only_all set (partial-step mode) the kernel
// does nothing unless every cell is active this step, the case k_limiter's
// list then skips.
template <typename R, int KH, int MINB>
__global__ void __launch_bounds__(128, MINB) k_limiter_st(int n, Params P, const Sched *__restrict__ S,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ lfj, const int2 *__restrict__ s12,
    const double4 *__restrict__ geo, const double4 *__restrict__ dr1, const unsigned char *__restrict__ fflag,
    const unsigned char *__restrict__ act, const double *__restrict__ tlast,
    const R *__restrict__ Wrec, R *__restrict__ tau, R *__restrict__ fst, const int *__restrict__ perm,
    const R *__restrict__ mnmx, const unsigned char *__restrict__ mz, int only_all, const R *__restrict__ lld) {
  constexpr int CST = limiter_cst<KH>();
  extern __shared__ __align__(16) unsigned char lsm[];
  __shared__ int soff[CST + 1];
  if (only_all && S->iscal[1] != n) return;
  const double t_global = S->t_global;
  const bool reuse = FVM_REUSE_MINMAX && S->mnmx_ok && S->iscal[1] == n;
  limiter_st_block<R, KH>(blockIdx.x, n, reuse, t_global, soff, lsm, off, lnk, lfj, s12, geo, dr1, fflag, act, tlast,
                          Wrec, tau, fst, perm, mnmx, mz, lld);
}
template <typename R, int KH, int MINB>
__global__ void __launch_bounds__(128, MINB) k_limiter(int n, Params P, const Sched *__restrict__ S,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ lfj, const int2 *__restrict__ s12,
    const double4 *__restrict__ geo, const double4 *__restrict__ dr1, const unsigned char *__restrict__ fflag,
    const unsigned char *__restrict__ act, const double *__restrict__ tlast,
    const R *__restrict__ Wrec, R *__restrict__ tau, R *__restrict__ fst, const int *__restrict__ perm,
    const R *__restrict__ mnmx, const unsigned char *__restrict__ mz, const int *__restrict__ clist,
    int skip_if_all, const R *__restrict__ lld) {
  if (skip_if_all && S->iscal[1] == n) return;  // the staged limiter has this step
  const double t_global = S->t_global;
  // every cell steps and every cell was reconstructed by the last step: the
  // neighbour min/max of pass 1 are the reconstruction's (same states, same
  // faces, exact min/max)
  const bool reuse = FVM_REUSE_MINMAX && S->mnmx_ok && S->iscal[1] == n;
  constexpr int TPC = 10 / KH;
  // TPC threads per cell; in partial steps a fixed grid strides over clist
  const long long cnt = (long long)TPC * (clist ? S->ninv : n);
  const bool lst = clist && S->ninv != n;  // every cell involved: the list is the identity
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cnt;
       t += (long long)gridDim.x * blockDim.x) {
    const int u = (int)(t / TPC);
    limiter_thread<R, KH>(lst ? clist[u] : perm[u], (int)(t % TPC) * KH, reuse, t_global, off, lnk, lfj, s12, geo,
                          dr1, fflag, act, tlast, Wrec, tau, fst, mnmx, mz, lld);
  }
}


// ---- compute_update face pass (MPI/compute_update.cpp:106-269) -----------
// One thread per face: half-step extrapolated face states, face velocity,
// rotated-frame HLLD flux.  Stores flux*dt*area, gradPsi and divB
// contributions (in the bulk type) for the owning cells to gather.
// Face flux of one pass under the learned-flux mode MODE: exact (LM_EXACT),
// exact with harvesting (LM_HARVEST), gate and defer to the network
// (LM_DEFER: returns false for a deferred face), or the deferred face's flux
// from the network output (LM_FINISH), falling back to the exact solver when
// the state either cell reaches from this face's flux alone over its step
// (tdt_i, tdt_j: area times each side's step) keeps less than half of its
// mass or of its thermal energy, or the result is not finite.
enum { LM_EXACT = 0, LM_HARVEST = 1, LM_DEFER = 2, LM_FINISH = 3 };

template <typename R, int MODE>
__device__ __forceinline__ bool learned_flux(const Params &P, const Sched *S, const LearnBuf &lb, int f, int slot,
                                             int pass, const R *wij, const R *Wi, const R *Wj, int jb, const R *nr,
                                             R &psi, R &Bn, R *flux, double tdt_i, double tdt_j, int i, int j) {
  if (MODE == LM_EXACT) {
    compute_flux<R>(P, wij, Wi, Wj, jb, nr, psi, Bn, flux);
    return true;
  }
  const unsigned salt = (unsigned)(S->steps * 2 + pass);
  if (MODE == LM_HARVEST) {
    HarvestSolver h{P, lb, (unsigned)f, salt};
    compute_flux_with<R>(P, wij, Wi, Wj, jb, nr, psi, Bn, flux, h);
    return true;
  }
  if (MODE == LM_DEFER) {
    DeferSolver h{P, lb, f};
    return compute_flux_with<R>(P, wij, Wi, Wj, jb, nr, psi, Bn, flux, h);
  }
  if (slot == 0) atomicAdd(&lb.stats[LSTAT_DEFERRED], (double)*lb.count);  // once per pass
  float y[8];
  const float4 *yp = reinterpret_cast<const float4 *>(lb.Y + 8 * (size_t)slot);
  const float4 y0 = yp[0], y1 = yp[1];
  y[0] = y0.x; y[1] = y0.y; y[2] = y0.z; y[3] = y0.w; y[4] = y1.x; y[5] = y1.y; y[6] = y1.z; y[7] = y1.w;
  LearnedSolver h{lb, y, lb.judge != 0 && face_hash((unsigned)f, salt) % lb.judge == 0};
  compute_flux_with<R>(P, wij, Wi, Wj, jb, nr, psi, Bn, flux, h);
  bool ok = true;
#pragma unroll
  for (int k = 0; k < NF; k++) ok = ok && isfinite(double(flux[k]));
  if (!ok) {
    compute_flux<R>(P, wij, Wi, Wj, jb, nr, psi, Bn, flux);
    atomicAdd(&lb.stats[LSTAT_FALLBACK], 1.0);
  } else if (!keeps_positive<R>(lb, i, -tdt_i, flux) || !keeps_positive<R>(lb, j, tdt_j, flux)) {
    compute_flux<R>(P, wij, Wi, Wj, jb, nr, psi, Bn, flux);
    atomicAdd(&lb.stats[LSTAT_FALLBACK], 1.0);
    atomicAdd(&lb.stats[LSTAT_POSFALL], 1.0);
  }
  return true;
}

template <typename R, int MODE>
__device__ __forceinline__ void corr_face(int f, int slot, double t_global, const Params &P, const Sched *__restrict__ S,
    const int2 *__restrict__ s12, const double4 *__restrict__ geo, const double4 *__restrict__ dr1,
    const unsigned char *__restrict__ fflag, const int *__restrict__ bnd, const double *__restrict__ vel,
    const double *__restrict__ tlast, const R *__restrict__ Wrec, const R *__restrict__ fst,
    R *__restrict__ fcon, unsigned char *__restrict__ fcode, const LearnBuf &lb) {
  const unsigned char ff = fflag[f];
  if (!(ff & FF_ACTIVE)) return;  // coded F_OFF with the flags
  const int2 e = s12[f];
  const double4 g = geo[f], d = dr1[f];
  R Wi[NF], Wj[NF];
  {  // issued with the face record, before the boundary tests
    const R *fs = fst + 20 * (size_t)f;
    load_n<R, NF>(fs, Wi);
    load_n<R, NF>(fs + 10, Wj);
  }
  int i = e.x, j = e.y;
  const double area = g.w;
  double nrm[3] = {g.x, g.y, g.z};
  double dri[3] = {d.x, d.y, d.z};
  unsigned char code = 0;
  if (ff & FF_BND1) {
    i = e.y; j = e.x;
    nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
    dri[0] = -dri[0]; dri[1] = -dri[1]; dri[2] = -dri[2];
    code |= F_SWAP;
  }
  const bool jbnd = (code & F_SWAP) ? (ff & FF_BND1) : (ff & FF_BND2);
  if (jbnd) code |= F_SKIPJ;
  const double dtI = t_global - tlast[i], dtJ = t_global - tlast[j];
  const double dt = smin(dtI, dtJ);
  const double dsh = d.w;  // (-dri).(-n) = dri.n
  if (jbnd) {  // the extrapolated states were not written for a boundary face: replaced, never used
    const R *ri = Wrec + 50 * (size_t)i;
#pragma unroll
    for (int k = 0; k < NF; k++) Wi[k] = Wj[k] = ri[k];
  }
  const double *vi = vel + 3 * (size_t)i, *vj = vel + 3 * (size_t)j;
  const double fij[3] = {dri[0] - nrm[0] * dsh, dri[1] - nrm[1] * dsh, dri[2] - nrm[2] * dsh};
  const double fdv = (vj[0] - vi[0]) * fij[0] + (vj[1] - vi[1]) * fij[1] + (vj[2] - vi[2]) * fij[2];
  const double ids2 = -0.5 * fdv * ((dsh > 0.0) ? 1.0 / sqr(dsh) : 0.0);
  const R wij[3] = {R((vj[0] + vi[0]) * 0.5 + dri[0] * ids2), R((vj[1] + vi[1]) * 0.5 + dri[1] * ids2),
                    R((vj[2] + vi[2]) * 0.5 + dri[2] * ids2)};
  const R nr[3] = {R(nrm[0]), R(nrm[1]), R(nrm[2])};
  R psi, Bn, flux[NF];
  const int jb = jbnd ? bnd[j] : NO_BOUNDARY;
  if (!learned_flux<R, MODE>(P, S, lb, f, slot, 0, wij, Wi, Wj, jb, nr, psi, Bn, flux, dt * area, dt * area, i, j)) {
    fcode[f] = code;  // deferred to the network; the contribution is written by the finishing pass
    return;
  }
  const double tarea = dt * area;
  R o[14];
#pragma unroll
  for (int k = 0; k < NF; k++) o[k] = R(double(flux[k]) * tarea);
  const double pt = double(psi) * tarea;
  o[10] = R(nrm[0] * pt); o[11] = R(nrm[1] * pt); o[12] = R(nrm[2] * pt);
  o[13] = R(double(Bn) * tarea);
  store_contrib<R>(fcon + 14 * (size_t)f, o);
  fcode[f] = code;
}

// One thread per face; in partial steps (use_list) a fixed grid strides over
// the active-face list, so a step with few active faces launches few blocks.
template <typename R, int MODE>
__global__ void __launch_bounds__(128, FVM_FLUX_MINB(R)) k_corr_flux(int nf, Params P, const Sched *__restrict__ S,
    const int2 *__restrict__ s12, const double4 *__restrict__ geo, const double4 *__restrict__ dr1,
    const unsigned char *__restrict__ fflag, const int *__restrict__ bnd, const double *__restrict__ vel,
    const double *__restrict__ tlast, const R *__restrict__ Wrec, const R *__restrict__ fst,
    R *__restrict__ fcon, unsigned char *__restrict__ fcode, LearnBuf lb, const int *__restrict__ flist,
    int use_list) {
  const double t_global = S->t_global;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (MODE == LM_FINISH) {  // one deferred face per thread
    if (t >= *lb.count) return;
    corr_face<R, MODE>(lb.gface[t], t, t_global, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec, fst, fcon, fcode, lb);
  } else if (use_list) {  // the active faces (the others were coded F_OFF with the flags)
    const int na = S->iscal[3];
    for (int u = t; u < na; u += gridDim.x * blockDim.x)  // the list is built only when some face is inactive
      corr_face<R, MODE>(na != nf ? flist[u] : u, -1, t_global, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec,
                         fst, fcon, fcode, lb);
  } else if (t < nf) {
    corr_face<R, MODE>(t, -1, t_global, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec, fst, fcon, fcode, lb);
  }
}

// The 14 contributions of face f as seven 2-wide loads (a face record is 112
// bytes in FP64 and 56 in FP32, so every record starts on a 16- or 8-byte
// boundary).
__device__ __forceinline__ void load_contrib(const double *o, double *v) {
  const double2 *o2 = reinterpret_cast<const double2 *>(o);
#pragma unroll
  for (int k = 0; k < 7; k++) { const double2 x = o2[k]; v[2 * k] = x.x; v[2 * k + 1] = x.y; }
}
__device__ __forceinline__ void load_contrib(const float *o, double *v) {
  const float2 *o2 = reinterpret_cast<const float2 *>(o);
#pragma unroll
  for (int k = 0; k < 7; k++) { const float2 x = o2[k]; v[2 * k] = x.x; v[2 * k + 1] = x.y; }
}

// Sum of the face contributions of cell c in its face order (the reference
// scatters in active-face order; both orders sum the same terms).  The FP32
// path accumulates its single-precision contributions in double with
// compensated (Kahan) summation.  A face's record is loaded before its code
// is tested and skipped faces add nothing (zero, or the Kahan state kept), so
// each face costs one dependent load after the link table and two faces'
// loads are in flight at once.
template <typename R>
__device__ __forceinline__ void gather_contrib(int c, int q0, int q1, const int2 *__restrict__ lfj,
                                               const R *__restrict__ fcon,
                                               const unsigned char *__restrict__ fcode, bool skipj_allowed,
                                               double *s) {
  constexpr bool kahan = sizeof(R) == 4;
  double comp[14];
#pragma unroll
  for (int k = 0; k < 14; k++) { s[k] = 0.0; comp[k] = 0.0; }
#pragma unroll 2
  for (int q = q0; q < q1; q++) {
    const int2 fj = lfj[q];
    const int f = fj.x;
    double v[14];
    load_contrib(fcon + 14 * (size_t)f, v);
    const unsigned char code = fcode[f];
    // this cell is the face's i side when it is s1 and the face was not
    // swapped, or s2 and it was
    const bool is_i = (fj.y >= 0) != ((code & F_SWAP) != 0);
    const bool use = !(code & F_OFF) && !(!is_i && skipj_allowed && (code & F_SKIPJ));
    // U: i gets -F, j gets +F;  gradPsi and divB: i gets +, j gets -
    // (a skipped face's record may hold anything, so it is never multiplied)
    const double wu = is_i ? -1.0 : 1.0;
#pragma unroll
    for (int k = 0; k < 14; k++) {
      if (kahan) {
        const double term = ((k < NF) == is_i) ? -v[k] : v[k];
        const double y = term - comp[k];
        const double t = s[k] + y;
        comp[k] = use ? (t - s[k]) - y : comp[k];
        s[k] = use ? t : s[k];
      } else {
        s[k] = fma(k < NF ? wu : -wu, use ? v[k] : 0.0, s[k]);  // exact: the weight is -1 or 1
      }
    }
  }
}

// ---- compute_update cell pass (MPI/compute_update.cpp:274-498) -----------
template <typename R>
__device__ __forceinline__ void corr_cell_body(int c, double t_global, const Params &P,
    const int *__restrict__ off, const int2 *__restrict__ lfj,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ tlast, double *__restrict__ volp,
    const R *__restrict__ Wrec, const R *__restrict__ tau,
    const R *__restrict__ fcon, const unsigned char *__restrict__ fcode,
    double *__restrict__ U, double *__restrict__ dU, double *__restrict__ stepdU,
    unsigned long long *__restrict__ counters, float *__restrict__ divb) {
  const unsigned char ac = act[c];
  if (!(ac & (A_ACTIVE | A_LNGB))) return;
  double s[14];
  gather_contrib<R>(c, off[c], off[c + 1], lfj, fcon, fcode, true, s);
  double *d0p = dU + 14 * (size_t)c;  // rows of 14 doubles: 2-wide loads and stores
  double d0[14];
  load_n<double, 14>(d0p, d0);
  const double zero14[14] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (!(ac & A_ACTIVE)) {
    // inactive neighbour: accumulate until its own step (collect_results,
    // MPI/distribute_work.cpp:714-720)
    if (stepdU) store_n<double, 14>(stepdU + 14 * (size_t)c, s);
    if (bnd[c] == NO_BOUNDARY) {
#pragma unroll
      for (int k = 0; k < NF; k++) d0[k] += s[k];
      d0[13] += s[13];
      d0[10] = d0[10] + s[10]; d0[11] = d0[11] + s[11]; d0[12] = d0[12] + s[12];
      store_n<double, 14>(d0p, d0);
    }
    return;
  }
  const double V = cvol[c];
  if (bnd[c] != NO_BOUNDARY) {
    volp[c] = V;
    store_n<double, 14>(d0p, zero14);
    if (stepdU) store_n<double, 14>(stepdU + 14 * (size_t)c, s);
    return;
  }
  double Uc[NF];
  load_n<double, NF>(U + 10 * (size_t)c, Uc);
#pragma unroll
  for (int k = 0; k < NF; k++) Uc[k] = Uc[k] + (d0[k] + s[k]);
  const double divB = d0[13] + s[13];
  const double dPsi[3] = {d0[10] + s[10], d0[11] + s[11], d0[12] + s[12]};
  const double dt = t_global - tlast[c];
  divb[c] = float(dt > 0.0 ? divB / dt / V : divB);  // divBi (MPI/distribute_work.cpp:681)
  store_n<double, 14>(d0p, zero14);  // dU_local = 0 (collect_results)
  if (stepdU) {
    double *sd = stepdU + 14 * (size_t)c;
#pragma unroll
    for (int k = 0; k < 13; k++) sd[k] = 0.0;
    sd[13] = dt > 0.0 ? divB / dt / V : divB;
  }
  R r[NF], rt[NF], tc[NF];  // w and t blocks of the record, tau
  load_n<R, NF>(Wrec + 50 * (size_t)c, r);
  load_n<R, NF>(Wrec + 50 * (size_t)c + 40, rt);
  load_n<R, NF>(tau + 10 * (size_t)c, tc);
  double W1[NF];
  if (Uc[MASS] <= 0.0) {
    // failed-mass fallback (MPI/compute_update.cpp:438-468)
    atomicAdd(&counters[0], 1ULL);
    double Ut[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) W1[k] = double(r[k]) + double(rt[k] * tc[k]) * dt;
    to_conservative(W1, volp[c], Ut);
    to_primitive(Ut, V, W1);
  } else {
    const double dth = 0.5 * dt;
    double Wh[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) Wh[k] = double(r[k]) + double(rt[k] * tc[k]) * dth;
    Uc[WBX] -= Wh[VELX] * divB;
    Uc[WBY] -= Wh[VELY] * divB;
    Uc[WBZ] -= Wh[VELZ] * divB;
    // Dedner divergence cleaning (MPI/compute_update.cpp:373-387, 403-405)
    const double pres = pressure(P, Wh);
    const double B2 = Wh[BX] * Wh[BX] + Wh[BY] * Wh[BY] + Wh[BZ] * Wh[BZ];
    const double dcs2 = P.gamma * pres + B2;
    const double ch_sig = sqrt(dcs2 / Wh[DENS]);
    Uc[WBX] -= dPsi[0];
    Uc[WBY] -= dPsi[1];
    Uc[WBZ] -= dPsi[2];
    Uc[MPSI] -= dcs2 * divB;
    const double l_min = pow(V / (4.0 * M_PI / 3.0), 1.0 / 3.0);
    Uc[MPSI] *= exp(-0.5 * ch_sig / l_min * dt);
    to_primitive(Uc, V, W1);
  }
  volp[c] = V;
  W1[ETHM] = ethm_update(P, W1, pos + 3 * (size_t)c);
  if (W1[ETHM] <= 0.0) {
    atomicAdd(&counters[1], 1ULL);
    W1[ETHM] = ethm_from_entropy(P, W1);
  } else {
    W1[ENTR] = entropy_from_ethm(P, W1);
  }
  double Un[NF];
  to_conservative(W1, V, Un);
  store_n<double, NF>(U + 10 * (size_t)c, Un);
}

// One thread per cell; in partial steps a fixed grid strides over the
// involved-cell list (clist, count ninv) instead of every cell.
template <typename R>
__global__ void __launch_bounds__(128) k_corr_cell(int n, Params P, const Sched *__restrict__ S,
    const int *__restrict__ off, const int2 *__restrict__ lfj, const int2 *__restrict__ s12,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ tlast, double *__restrict__ volp,
    const R *__restrict__ Wrec, const R *__restrict__ tau,
    const R *__restrict__ fcon, const unsigned char *__restrict__ fcode,
    double *__restrict__ U, double *__restrict__ dU, double *__restrict__ stepdU,
    unsigned long long *__restrict__ counters, const int *__restrict__ perm, float *__restrict__ divb,
    const int *__restrict__ clist) {
  const double t_global = S->t_global;
  const int cnt = clist ? S->ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x)
    corr_cell_body<R>(lst ? clist[t] : perm[t], t_global, P, off, lfj, cvol, act, bnd, pos, tlast, volp, Wrec, tau,
                      fcon, fcode, U, dU, stepdU, counters, divb);
}

// ---- compute_pvel (MPI/compute_pvel.cpp:5-52) -----------------------------
__device__ __forceinline__ void pvel_body(int i, const Params &P, const unsigned char *__restrict__ act,
                       const int *__restrict__ bnd,
                       const double *__restrict__ U, const double *__restrict__ volp,
                       const double *__restrict__ cvol, const double *__restrict__ ccen,
                       const double *__restrict__ pos, double *__restrict__ vel) {
  if (!(act[i] & A_ACTIVE)) return;
  if (P.static_mesh) {  // compute_pvel1 hook returning true (MPI/set_problem.cpp:61-72)
    double *vo = vel + 3 * (size_t)i;
    vo[0] = vo[1] = vo[2] = 0.0;
    return;
  }
  double W[NF];
  to_primitive(U + 10 * (size_t)i, volp[i], W);
  double v[3] = {W[VELX], W[VELY], W[VELZ]};
  const double B2 = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
  const double cs2 = (P.gamma * pressure(P, W) + B2) / W[DENS];
  const double vel2 = W[VELX] * W[VELX] + W[VELY] * W[VELY] + W[VELZ] * W[VELZ];
  const double vabs = sqrt(cs2 + vel2);
  const double *cc = ccen + 3 * (size_t)i, *x = pos + 3 * (size_t)i;
  const double d3[3] = {cc[0] - x[0], cc[1] - x[1], cc[2] - x[2]};
  const double d = sqrt(d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2]);
  if (d != 0.0) {
    const double eta = 0.25f, ki = 1.0f, f1 = 0.9f, f2 = 1.1f;
    const double R = pow(cvol[i] * (3.0 / (4.0 * M_PI)), 1.0 / 3.0);
    const double fac = d / (eta * R);
    double f;
    if (fac < f1) f = 0.0;
    else if (fac < f2) f = (d - f1 * eta * R) / ((f2 - f1) * eta * R);
    else f = 1.0;
    const double tau = d / vabs;
    f *= ki / tau;
    v[0] += d3[0] * f; v[1] += d3[1] * f; v[2] += d3[2] * f;
    if (bnd[i] != NO_BOUNDARY) v[0] = v[1] = v[2] = 0.0;
  }
  double *vo = vel + 3 * (size_t)i;
  vo[0] = v[0]; vo[1] = v[1]; vo[2] = v[2];
}

// Every cell, or in partial steps the involved-cell list.
__global__ void k_pvel(int n, Params P, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
                       const double *__restrict__ U, const double *__restrict__ volp,
                       const double *__restrict__ cvol, const double *__restrict__ ccen,
                       const double *__restrict__ pos, double *__restrict__ vel, const int *__restrict__ clist,
                       const int *__restrict__ ninv) {
  const int cnt = clist ? *ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x)
    pvel_body(lst ? clist[t] : t, P, act, bnd, U, volp, cvol, ccen, pos, vel);
}

// ---- compute_timestep(i) (MPI/compute_timestep.cpp:6-51) ------------------
// The face minimum min_f h / x_f is taken as h / max_f x_f: h > 0 and a
// rounded quotient never increases with its divisor, so both give the same
// double, with one division instead of one per face.
__device__ double cell_timestep(const Params &P, int i, bool with_faces, const int *off, const int2 *lfj,
                                const int *bnd, const double *U, const double *volp, const double *vel) {
  double W[NF];
  to_primitive(U + 10 * (size_t)i, volp[i], W);
  const double *pv = vel + 3 * (size_t)i;
  double csi = 0.0, vrel = 0.0;
  const bool b = bnd[i] != NO_BOUNDARY;
  if (!b) {
    const double Pi = pressure(P, W) * P.gamma;
    const double B2i = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
    csi = sqrt((Pi + B2i) / W[DENS]);
    const double s = with_faces ? 1.0 : 0.0;
    const double d[3] = {W[VELX] - pv[0] * s, W[VELY] - pv[1] * s, W[VELZ] - pv[2] * s};
    vrel = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  }
  const double h = pow(volp[i] / (4.0 * M_PI / 3.0), 1.0 / 3.0);
  double dti = h / (csi + vrel + 1.0 / FVM_HUGE);
  if (with_faces) {
    const double fac = b ? 0.0 : 1.0;
    double xmax = 0.0;
    const int q1 = off[i + 1];
    for (int q = off[i]; q < q1; q++) {
      const int2 fj = lfj[q];
      const int j = fj.y >= 0 ? fj.y : ~fj.y;
      const double *vj = vel + 3 * (size_t)j;
      const double w3[3] = {(vj[0] + pv[0]) * 0.5, (vj[1] + pv[1]) * 0.5, (vj[2] + pv[2]) * 0.5};
      const double dw[3] = {vj[0] - pv[0], vj[1] - pv[1], vj[2] - pv[2]};
      const double r[3] = {W[VELX] - w3[0], W[VELY] - w3[1], W[VELZ] - w3[2]};
      const double rv = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const double dwa = sqrt(dw[0] * dw[0] + dw[1] * dw[1] + dw[2] * dw[2]);
      xmax = smax(xmax, smax(fac * (csi + rv), 1.0 / FVM_HUGE + dwa));
    }
    if (q1 > off[i]) dti = smin(dti, h / xmax);
  }
  return dti * P.courant;
}

__device__ __forceinline__ double extra_timestep(const Params &P, int i, const int *bnd, const double *pos,
                                                 const double *vel) {
  if (P.eos == 0 || bnd[i] != NO_BOUNDARY) return FVM_HUGE;
  const double *x = pos + 3 * (size_t)i, *v = vel + 3 * (size_t)i;
  const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  return P.courant * r / (1.0 / FVM_HUGE + sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
}

__device__ __forceinline__ void atomic_min_pos(double *addr, double v) {
  atomicMin((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// compute_timesteps(false) first loops (MPI/compute_timestep.cpp:78-96); the
// global minimum is reduced per warp before one atomic per warp
__global__ void k_timestep(int n, Params P, const int *__restrict__ off, const int2 *__restrict__ lfj,
                           const unsigned char *__restrict__ act,
                           const int *__restrict__ bnd, const double *__restrict__ U,
                           const double *__restrict__ volp, const double *__restrict__ vel,
                           const double *__restrict__ pos, const double *__restrict__ tlast,
                           const double *__restrict__ tend, double *__restrict__ dtl,
                           double *__restrict__ dmin, const int *__restrict__ clist, const int *__restrict__ ninv) {
  // every cell, or in partial steps the involved-cell list (the dt of any
  // other cell is never read)
  double vmin = FVM_HUGE;
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = blockIdx.x * blockDim.x + threadIdx.x; t_ < cnt_; t_ += gridDim.x * blockDim.x) {
    const int i = lst ? clist[t_] : t_;
    const unsigned char a = act[i];
    if (!(a & (A_ACTIVE | A_LNGB))) {
      dtl[i] = FVM_HUGE;
    } else if (!(a & A_ACTIVE)) {
      dtl[i] = (tend[i] - tlast[i]) * (bnd[i] != NO_BOUNDARY ? -1.0 : 1.0);
    } else {
      const double dti = smin(extra_timestep(P, i, bnd, pos, vel),
                              cell_timestep(P, i, true, off, lfj, bnd, U, volp, vel));
      vmin = smin(vmin, dti);
      dtl[i] = bnd[i] != NO_BOUNDARY ? -1.0 * dti : dti;
    }
  }
  for (int o = 16; o > 0; o >>= 1) vmin = smin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0 && vmin < FVM_HUGE) atomic_min_pos(dmin, vmin);
}

// dt >= 8 dt_min halving (MPI/compute_timestep.cpp:103-104)
__global__ void k_halve(int n, const unsigned char *__restrict__ act, const double *__restrict__ dmin,
                        double *__restrict__ dtl, const int *__restrict__ clist, const int *__restrict__ ninv) {
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = blockIdx.x * blockDim.x + threadIdx.x; t_ < cnt_; t_ += gridDim.x * blockDim.x) {
    const int i = lst ? clist[t_] : t_;
    if ((act[i] & A_ACTIVE) && dtl[i] >= 8.0 * dmin[0]) dtl[i] *= 0.5;
  }
}

// adjust_timesteps relaxation (MPI/compute_timestep.cpp:123-142).  The
// reference relaxes neighbour pairs sequentially in site order and the result
// depends on that order.  Exact reproduction in three parts:
//  1. k_adjust_mark (parallel): hash marks, which do not depend on the order,
//     and a count of "dirty" sites, active sites with a neighbour whose dt is
//     outside a factor 2 of their own;
//  2. with no dirty site every pair already satisfies the bound, no value
//     changes, and the sweep is skipped;
//  3. otherwise k_adjust_seq sweeps the ascending list of active
//     non-boundary sites (compacted in parallel) in one thread, exactly as
//     the reference does.
__global__ void k_adjust_mark(int n, const int *__restrict__ off, const int2 *__restrict__ lfj,
                              const unsigned char *__restrict__ act,
                              const int *__restrict__ bnd, const double *__restrict__ dtl,
                              unsigned char *__restrict__ hash, int *__restrict__ ndirty,
                              unsigned char *__restrict__ site, unsigned char *__restrict__ work,
                              const int *__restrict__ clist, const int *__restrict__ ninv) {
  // site[] starts cleared; only the active non-boundary sites are marked
  int ndirty_t = 0;
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = blockIdx.x * blockDim.x + threadIdx.x; t_ < cnt_; t_ += gridDim.x * blockDim.x) {
    const int i = lst ? clist[t_] : t_;
    if (!(act[i] & A_ACTIVE) || bnd[i] != NO_BOUNDARY) continue;
    bool dirty = false;
    site[i] = 1;
    const double di = dtl[i];
    for (int q = off[i]; q < off[i + 1]; q++) {
      const int2 fj = lfj[q];
      const int j = fj.y >= 0 ? fj.y : ~fj.y;
      const double dj = dtl[j];
      if (dj < 0.0) continue;
      hash[j] = 1;
      if (2.0 * dj < di || 2.0 * di < dj) {
        dirty = true;
        work[j] = 1;  // both ends of a pair outside a factor 2 start the replay's work list
      }
    }
    if (dirty) { work[i] = 1; ndirty_t++; }
  }
  __shared__ int bsum;
  if (threadIdx.x == 0) bsum = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) ndirty_t += __shfl_xor_sync(0xffffffffu, ndirty_t, o);
  if ((threadIdx.x & 31) == 0 && ndirty_t) atomicAdd(&bsum, ndirty_t);
  __syncthreads();
  if (threadIdx.x == 0 && bsum) atomicAdd(ndirty, bsum);
}

// Order-preserving compaction of flagged cells: per-block counts, one-block
// exclusive scan of the counts, then per-block placement.
constexpr int CB = 1024;
__global__ void k_count_flags(int n, const unsigned char *__restrict__ flag, int *__restrict__ bcount) {
  const int i = blockIdx.x * CB + threadIdx.x;
  const bool v = i < n && flag[i];
  __shared__ int bs;
  if (threadIdx.x == 0) bs = 0;
  __syncthreads();
  const unsigned cnt = __popc(__ballot_sync(0xffffffffu, v));
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&bs, (int)cnt);
  __syncthreads();
  if (threadIdx.x == 0) bcount[blockIdx.x] = bs;
}
__global__ void k_scan_counts(int nb, int *__restrict__ bcount, int *__restrict__ total) {
  // one block of CB threads, each summing ceil(nb / CB) consecutive counts
  __shared__ int part[CB];
  const int per = (nb + CB - 1) / CB;
  const int b0 = threadIdx.x * per;
  int sum = 0;
  for (int b = b0; b < b0 + per && b < nb; b++) sum += bcount[b];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < CB; o <<= 1) {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - sum;  // exclusive prefix of this thread's range
  for (int b = b0; b < b0 + per && b < nb; b++) {
    const int c = bcount[b];
    bcount[b] = run;
    run += c;
  }
  if (threadIdx.x == CB - 1) *total = part[CB - 1];
}
__global__ void k_place_flags(int n, const unsigned char *__restrict__ flag, const int *__restrict__ boff,
                              int *__restrict__ list) {
  const int i = blockIdx.x * CB + threadIdx.x;
  const bool v = i < n && flag[i];
  __shared__ int wsum[CB / 32];
  const unsigned b = __ballot_sync(0xffffffffu, v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(b);
  __syncthreads();
  int base = boff[blockIdx.x];
  for (int k = 0; k < w; k++) base += wsum[k];
  if (v) list[base + __popc(b & ((1u << lane) - 1u))] = i;
}

// Ordered placement of the active faces (fflag & FF_ACTIVE), from the
// per-block counts k_faceflags writes and their scan; a no-op when every face
// is active, where the flux passes map threads to faces directly.
__global__ void k_place_faces(int nf, const unsigned char *__restrict__ fflag, const int *__restrict__ nactive,
                              const int *__restrict__ boff, int *__restrict__ list) {
  if (*nactive == nf) return;
  const int i = blockIdx.x * CB + threadIdx.x;
  const bool v = i < nf && (fflag[i] & FF_ACTIVE);
  __shared__ int wsum[CB / 32];
  const unsigned b = __ballot_sync(0xffffffffu, v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(b);
  __syncthreads();
  int base = boff[blockIdx.x];
  for (int k = 0; k < w; k++) base += wsum[k];
  if (v) list[base + __popc(b & ((1u << lane) - 1u))] = i;
}

// The cells a partial step works on (active, or inactive neighbours of
// active cells), in index order.
__global__ void k_count_cells(int n, const unsigned char *__restrict__ act, int *__restrict__ bcount) {
  const int i = blockIdx.x * CB + threadIdx.x;
  const bool v = i < n && (act[i] & (A_ACTIVE | A_LNGB));
  __shared__ int bs;
  if (threadIdx.x == 0) bs = 0;
  __syncthreads();
  const unsigned cnt = __popc(__ballot_sync(0xffffffffu, v));
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&bs, (int)cnt);
  __syncthreads();
  if (threadIdx.x == 0) bcount[blockIdx.x] = bs;
}
__global__ void k_place_cells(int n, const unsigned char *__restrict__ act, const int *__restrict__ boff,
                              int *__restrict__ list) {
  const int i = blockIdx.x * CB + threadIdx.x;
  const bool v = i < n && (act[i] & (A_ACTIVE | A_LNGB));
  __shared__ int wsum[CB / 32];
  const unsigned b = __ballot_sync(0xffffffffu, v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(b);
  __syncthreads();
  int base = boff[blockIdx.x];
  for (int k = 0; k < w; k++) base += wsum[k];
  if (v) list[base + __popc(b & ((1u << lane) - 1u))] = i;
}

__global__ void k_adjust_seq(const int *__restrict__ off, const int *__restrict__ lnk,
                             const int2 *__restrict__ s12, const int *__restrict__ alist,
                             const int *__restrict__ nsite, const int *__restrict__ ndirty,
                             double *__restrict__ dtl) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (*ndirty == 0) return;  // nonzero when the sweep must run
  const int m = *nsite;
  for (int a = 0; a < m; a++) {
    const int i = alist[a];
    double di = dtl[i];
    for (int q = off[i]; q < off[i + 1]; q++) {
      const int2 e = s12[lnk[q]];
      const int j = e.x == i ? e.y : e.x;
      double dj = dtl[j];
      if (dj < 0.0) continue;
      di = smin(di, 2.0 * dj);
      dj = smin(dj, 2.0 * di);
      dtl[j] = dj;
      dtl[i] = di;
    }
  }
}

// ---- adjust_timesteps in parallel, bit for bit ----------------------------
// The sequential sweep above visits the active non-boundary sites in
// ascending order; at site i, for each face slot in order with a non-boundary
// neighbour j, it sets dt_i = min(dt_i, 2 dt_j) and then
// dt_j = min(dt_j, 2 dt_i).  min and doubling are exact, so every value the
// sweep produces is 2^k dt0_y for a chain of such updates that runs forward in
// sweep order, and each final dt is the minimum over the chains that end at
// it.  The kernels below compute that minimum as a fixed point.  Per link q
// (cell u, face slot s, neighbour v) they keep
//   rdv[q]: dt of v when the sweep reaches u's slot s (what u reads there),
//   wrv[q]: dt of u just after its own update at slot s (what v then reads).
// Each replay lets every involved site walk its own timeline: the slots of
// its active neighbours at their positions in the order (the sweep reads the
// site's dt, then lowers it) and, for an active site, its own slots at its
// own position.  It reads the neighbours' entries, writes its own, and keeps
// the result in dtl.  Entries only decrease and start at the initial dt, an
// upper bound, so replays converge; a replay that changes nothing leaves the
// exact result.  Replays after convergence return at once.  If ADJ_ITERS
// replays have not settled, the sequential sweep runs from the initial dt.
// A site's outputs are a function of its own initial dt and the entries it
// reads, and equal their initial values while it is within a factor 2 of
// every neighbour, so each replay walks only a work list: the ends of
// out-of-bound pairs in the first, afterwards the sites whose entries the
// previous replay lowered (awork, two alternating bytes per cell).
// aflag[0..2]: changed flags of replays k % 3; [3] replays run; [4] fallback;
// [5] settled (or nothing to do).
constexpr int ADJ_ITERS = 24;

__device__ __forceinline__ int lfj_nb(int2 fj) { return fj.y >= 0 ? fj.y : ~fj.y; }

__global__ void k_adjust_init(int n, const int *__restrict__ off, const int2 *__restrict__ lfj,
                              const unsigned char *__restrict__ act, const int *__restrict__ ndirty,
                              const double *__restrict__ dtl, double *__restrict__ dt0, double *__restrict__ rdv,
                              double *__restrict__ wrv, int *__restrict__ aflag, const int *__restrict__ clist,
                              const int *__restrict__ ninv) {
  if (*ndirty == 0) return;  // every pair is within a factor 2: nothing changes
  if (blockIdx.x == 0 && threadIdx.x == 0) aflag[2] = 1;  // replay 0 runs
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = blockIdx.x * blockDim.x + threadIdx.x; t_ < cnt_; t_ += gridDim.x * blockDim.x) {
    const int u = lst ? clist[t_] : t_;
    if (!(act[u] & (A_ACTIVE | A_LNGB))) continue;
    const double du = dtl[u];
    dt0[u] = du;
    for (int q = off[u]; q < off[u + 1]; q++) {
      const int v = lfj_nb(lfj[q]);
      rdv[q] = (act[v] & (A_ACTIVE | A_LNGB)) ? dtl[v] : du;
      wrv[q] = du;
    }
  }
}

__global__ void k_adjust_replay(int n, int kparam, const int *__restrict__ off, const int2 *__restrict__ lfj,
                                const int *__restrict__ lsort, const int *__restrict__ lpart,
                                const unsigned char *__restrict__ act, const double *__restrict__ dt0,
                                double *__restrict__ rdv, double *__restrict__ wrv, double *__restrict__ dtl,
                                int *__restrict__ aflag, unsigned char *__restrict__ work, int kdev) {
  // replay index: the launch's, or (in a captured step) aflag[7], which
  // k_adjust_next advances between replays
  const int k = kdev ? aflag[7] : kparam;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (aflag[5]) return;
  if (aflag[(k + 2) % 3] == 0) {  // the previous replay changed nothing (or none was needed)
    if (t0 == 0) aflag[5] = 1;
    return;
  }
  if (t0 == 0) { aflag[(k + 1) % 3] = 0; aflag[3] += 1; }
  bool changed = false;
  unsigned char *cur = work + (size_t)(k & 1) * n, *nxt = work + (size_t)((k + 1) & 1) * n;
  for (int u = t0; u < n; u += gridDim.x * blockDim.x) {  // grid-stride: a settled replay costs one launch
    if (!cur[u]) continue;  // inputs unchanged since u was last walked
    cur[u] = 0;
    const unsigned char a = act[u];
    if (!(a & (A_ACTIVE | A_LNGB))) continue;
    const double d0 = dt0[u];
    if (d0 < 0.0) continue;  // boundary: neither swept nor relaxed
    const bool swept = (a & A_ACTIVE) != 0;
    const int q0 = off[u], q1 = off[u + 1];
    double dtu = d0;
    bool own_done = !swept;
    auto own_slots = [&]() {  // the sweep at u's own position
      for (int q = q0; q < q1; q++) {
        const int v = lfj_nb(lfj[q]);
        if (dt0[v] < 0.0) continue;
        dtu = smin(dtu, 2.0 * rdv[q]);
        if (dtu < wrv[q]) { wrv[q] = dtu; changed = true; nxt[v] = 1; }
      }
    };
    for (int t = q0; t < q1; t++) {  // neighbours in ascending index = sweep order
      const int q = lsort[t];
      const int v = lfj_nb(lfj[q]);
      if (!own_done && v > u) { own_slots(); own_done = true; }
      if ((act[v] & A_ACTIVE) && dt0[v] >= 0.0) {  // the sweep at v's position, v's slot for this face
        const int p = lpart[q];
        if (dtu < rdv[p]) { rdv[p] = dtu; changed = true; nxt[v] = 1; }
        dtu = smin(dtu, 2.0 * wrv[p]);
      }
    }
    if (!own_done) own_slots();
    dtl[u] = dtu;
  }
  if (changed) aflag[k % 3] = 1;
}

// In a captured step the replays run as the body of a conditional WHILE
// node: after replay k this single thread stops the loop once replay k
// changed nothing (settled) or ADJ_ITERS replays have run, and advances k.
__global__ void k_adjust_next(int *__restrict__ aflag, cudaGraphConditionalHandle loop) {
  const int k = aflag[7];
  bool stop = aflag[5] != 0;
  if (aflag[k % 3] == 0) { aflag[5] = 1; stop = true; }
  if (k + 1 >= ADJ_ITERS) stop = true;
  aflag[7] = k + 1;
  cudaGraphSetConditional(loop, stop ? 0u : 1u);
}

// Not settled after ADJ_ITERS replays: restore the initial dt for the
// sequential sweep.
__global__ void k_adjust_restore(int n, const unsigned char *__restrict__ act, const double *__restrict__ dt0,
                                 double *__restrict__ dtl, int *__restrict__ aflag, int *__restrict__ stats,
                                 const int *__restrict__ clist, const int *__restrict__ ninv) {
  const bool fallback = !aflag[5] && aflag[(ADJ_ITERS - 1) % 3] != 0;
  const bool first = blockIdx.x == 0 && threadIdx.x == 0;
  if (first) { stats[0] = aflag[3]; stats[1] = fallback ? 1 : 0; }
  if (!fallback) return;
  if (first) aflag[4] = 1;
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = blockIdx.x * blockDim.x + threadIdx.x; t_ < cnt_; t_ += gridDim.x * blockDim.x) {
    const int u = lst ? clist[t_] : t_;
    if (act[u] & (A_ACTIVE | A_LNGB)) dtl[u] = dt0[u];
  }
}

// rung assignment and inactive-neighbour promotion (MPI/compute_timestep.cpp
// :144-199) fused with collect_results (MPI/distribute_work.cpp:676-713) and
// the tlast/tend update of correct() (set_problem.cpp generic hook)
template <typename R>
__device__ __forceinline__ void rungs_body(int i, double t_global, int min_rung, const Params &P, int shared,
                        const unsigned char *__restrict__ act, const unsigned char *__restrict__ hash,
                        const double *__restrict__ dtl, const double *__restrict__ dmin,
                        int *__restrict__ rung, double *__restrict__ tlast, double *__restrict__ tend,
                        R *__restrict__ Wrec, int *__restrict__ iscal, const double *__restrict__ vel,
                        double *__restrict__ opos, double *__restrict__ ovel) {
  const unsigned char a = act[i];
  if (!(a & (A_ACTIVE | A_LNGB))) return;
  if (a & A_ACTIVE) {
    const int r = shared ? get_rung(P, dmin[0], min_rung) : get_rung(P, fabs(dtl[i]), min_rung);
    rung[i] = r;
    // correct() (MPI/set_problem.cpp:89-101): generator motion over the step
    const double dth = 0.5 * (t_global - tlast[i]);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double v = vel[3 * (size_t)i + a];
      opos[3 * (size_t)i + a] = opos[3 * (size_t)i + a] + (v + ovel[3 * (size_t)i + a]) * dth;
      ovel[3 * (size_t)i + a] = v;
    }
    tlast[i] = t_global;
    tend[i] = t_global + get_dt(P, r);
    if (r < 0 || r >= RUNGMAX) atomicOr(&iscal[2], 1);
    return;
  }
  if (shared || !hash[i]) return;
  const double tl = tlast[i], te = tend[i];
  if (tl == t_global) return;
  if (!(te - tl > dtl[i])) return;
  const int rr = smax(exp_of(P.dtmax) - exp_of(fabs(0.5 * dtl[i])), 0);
  const double dt = get_dt(P, rr);
  int rn;
  double tn;
  if (tl + dt <= t_global) {
    rn = get_rung(P, dt, min_rung);
    tn = t_global + get_dt(P, rn);
    rn = -1 - rn;
  } else {
    rn = rr;
    tn = tl + dt;
  }
  if (tn - tl < te - tl) {
    rung[i] = rn < 0 ? -1 - rn : rn;
    tend[i] = tn;
    if (rn < 0) {
      R *w = Wrec + 50 * (size_t)i;
      for (int k = 10; k < 50; k++) w[k] = R(0);
    }
  }
}

// Every cell, or in partial steps the involved-cell list.
template <typename R>
__global__ void k_rungs(int n, Params P, const Sched *__restrict__ S, int shared,
                        const unsigned char *__restrict__ act, const unsigned char *__restrict__ hash,
                        const double *__restrict__ dtl, const double *__restrict__ dmin,
                        int *__restrict__ rung, double *__restrict__ tlast, double *__restrict__ tend,
                        R *__restrict__ Wrec, int *__restrict__ iscal, const double *__restrict__ vel,
                        double *__restrict__ opos, double *__restrict__ ovel, const int *__restrict__ clist) {
  const double t_global = S->t_global;
  const int min_rung = S->min_rung;
  const int cnt = clist ? S->ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x)
    rungs_body<R>(lst ? clist[t] : t, t_global, min_rung, P, shared, act, hash, dtl, dmin, rung, tlast, tend, Wrec,
                  iscal, vel, opos, ovel);
}

// distribute_fluid_update_data: primitives of the updated state
template <typename R>
__global__ void k_wst(int n, const unsigned char *__restrict__ act, const double *__restrict__ U,
                      const double *__restrict__ volp, R *__restrict__ Wst, const int *__restrict__ clist,
                      const int *__restrict__ ninv) {
  const int cnt = clist ? *ninv : n;  // every cell, or in partial steps the involved-cell list
  const bool lst = clist && cnt != n;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
    const int i = lst ? clist[t] : t;
    if (!(act[i] & (A_ACTIVE | A_LNGB))) continue;
    double u[NF], W[NF];
    load_n<double, NF>(U + 10 * (size_t)i, u);
    to_primitive(u, volp[i], W);
    R w[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) w[k] = R(W[k]);
    store_n<R, NF>(Wst + 10 * (size_t)i, w);
  }
}

// ---- compute_update0 face pass (MPI/compute_update.cpp:713-810) ----------
template <typename R, int MODE>
__device__ __forceinline__ void pred_face(int f, int slot, const Params &P,
    const int2 *__restrict__ s12, const double4 *__restrict__ geo, const double4 *__restrict__ dr1,
    const unsigned char *__restrict__ fflag, const int *__restrict__ bnd,
    const double *__restrict__ vel, const R *__restrict__ Wst,
    R *__restrict__ fcon, unsigned char *__restrict__ fcode, const Sched *__restrict__ S, const int *__restrict__ rung,
    const LearnBuf &lb) {
  const unsigned char ff = fflag[f];
  if (!(ff & FF_ACTIVE)) return;  // coded F_OFF with the flags
  const int2 e = s12[f];
  int i = e.x, j = e.y;
  const double4 g = geo[f], d = dr1[f];
  const double area = g.w;
  double nrm[3] = {g.x, g.y, g.z};
  double dri[3] = {d.x, d.y, d.z};
  unsigned char code = 0;
  bool ib = ff & FF_BND1, jbf = ff & FF_BND2;
  if (ib) {
    i = e.y; j = e.x;
    nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
    dri[0] = -dri[0]; dri[1] = -dri[1]; dri[2] = -dri[2];
    code |= F_SWAP;
    const bool tmp = ib; ib = jbf; jbf = tmp;
  }
  if (ib) { fcode[f] = F_OFF; return; }
  const int jb = jbf ? bnd[j] : NO_BOUNDARY;
  const double dsh = d.w;
  R Wi[NF], Wj[NF];
  const R *wi = Wst + 10 * (size_t)i, *wj = Wst + 10 * (size_t)(jb == NO_BOUNDARY ? j : i);
  load_n<R, NF>(wi, Wi);
  load_n<R, NF>(wj, Wj);
  const double *vi = vel + 3 * (size_t)i, *vj = vel + 3 * (size_t)j;
  const double fij[3] = {dri[0] - nrm[0] * dsh, dri[1] - nrm[1] * dsh, dri[2] - nrm[2] * dsh};
  const double fdv = (vj[0] - vi[0]) * fij[0] + (vj[1] - vi[1]) * fij[1] + (vj[2] - vi[2]) * fij[2];
  const double ids2 = -0.5 * fdv * ((dsh > 0.0) ? 1.0 / sqr(dsh) : 0.0);
  const R wij[3] = {R((vj[0] + vi[0]) * 0.5 + dri[0] * ids2), R((vj[1] + vi[1]) * 0.5 + dri[1] * ids2),
                    R((vj[2] + vi[2]) * 0.5 + dri[2] * ids2)};
  const R nr[3] = {R(nrm[0]), R(nrm[1]), R(nrm[2])};
  R psi, Bn, flux[NF];
  {
    // positivity horizon of each side: its own step dt(rung)
    const double ai = MODE == LM_FINISH ? area * get_dt(P, rung[i]) : 0.0;
    const double aj = MODE == LM_FINISH ? area * get_dt(P, rung[j]) : 0.0;
    if (!learned_flux<R, MODE>(P, S, lb, f, slot, 1, wij, Wi, Wj, jb, nr, psi, Bn, flux, ai, aj, i, j)) {
      fcode[f] = code;
      return;
    }
  }
  R o[14];
#pragma unroll
  for (int k = 0; k < NF; k++) o[k] = R(double(flux[k]) * area);
  const double pa2 = double(psi) * area;
  o[10] = R(nrm[0] * pa2); o[11] = R(nrm[1] * pa2); o[12] = R(nrm[2] * pa2);
  o[13] = R(double(Bn) * area);
  store_contrib<R>(fcon + 14 * (size_t)f, o);
  fcode[f] = code;
}

// One thread per face; a fixed grid strides over the active-face list in
// partial steps (see k_corr_flux).
template <typename R, int MODE>
__global__ void __launch_bounds__(128, FVM_FLUX_MINB(R)) k_pred_flux(int nf, Params P,
    const int2 *__restrict__ s12, const double4 *__restrict__ geo, const double4 *__restrict__ dr1,
    const unsigned char *__restrict__ fflag, const int *__restrict__ bnd,
    const double *__restrict__ vel, const R *__restrict__ Wst,
    R *__restrict__ fcon, unsigned char *__restrict__ fcode, const Sched *__restrict__ S, const int *__restrict__ rung,
    LearnBuf lb, const int *__restrict__ flist, int use_list) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (MODE == LM_FINISH) {
    if (t >= *lb.count) return;
    pred_face<R, MODE>(lb.gface[t], t, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb);
  } else if (use_list) {
    const int na = S->iscal[3];
    for (int u = t; u < na; u += gridDim.x * blockDim.x)
      pred_face<R, MODE>(na != nf ? flist[u] : u, -1, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb);
  } else if (t < nf) {
    pred_face<R, MODE>(t, -1, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb);
  }
}

// ---- compute_update0 cell pass + collect_reconstruction -------------------
// (MPI/compute_update.cpp:812-964; MPI/distribute_work.cpp:820-834)
// Writes the predicted time derivative t into the cell's Wrec and the
// cell's final rung/tend.  Arithmetic in double for both bulk types.
template <typename R>
__device__ __forceinline__ void pred_cell_body(int c, double t_global, int min_rung, const Params &P,
    const int *__restrict__ off, const int2 *__restrict__ lfj,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ U,
    const R *__restrict__ fcon, const unsigned char *__restrict__ fcode,
    int *__restrict__ rung, double *__restrict__ tend, R *__restrict__ Wrec) {
  if (!(act[c] & A_ACTIVE) || bnd[c] != NO_BOUNDARY) return;
  const double V = cvol[c];
  double dot[14];
  gather_contrib<R>(c, off[c], off[c + 1], lfj, fcon, fcode, false, dot);
  double u0[NF], W0[NF];
  load_n<double, NF>(U + 10 * (size_t)c, u0);
  to_primitive(u0, V, W0);
  int rg = rung[c];
  while (rg < RUNGMAX - 1 && u0[MASS] + dot[MASS] * get_dt(P, rg) <= 0.0 * u0[MASS]) rg++;
  const double dt = get_dt(P, rg);
  double Uc[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) Uc[k] = u0[k] + dot[k] * dt;
  {
    const double divB = dot[13];
    Uc[WBX] -= W0[VELX] * divB * dt;
    Uc[WBY] -= W0[VELY] * divB * dt;
    Uc[WBZ] -= W0[VELZ] * divB * dt;
    const double pres = pressure(P, W0);
    const double B2 = W0[BX] * W0[BX] + W0[BY] * W0[BY] + W0[BZ] * W0[BZ];
    const double dcs2 = P.gamma * pres + B2;
    const double ch_sig = sqrt(dcs2 / W0[DENS]);
    Uc[WBX] -= dot[10] * dt;
    Uc[WBY] -= dot[11] * dt;
    Uc[WBZ] -= dot[12] * dt;
    Uc[MPSI] -= dcs2 * divB * dt;
    const double l_min = pow(V / (4.0 * M_PI / 3.0), 1.0 / 3.0);
    Uc[MPSI] *= exp(-0.5 * ch_sig / l_min * dt);
  }
  double W1[NF];
  to_primitive(Uc, V, W1);
  W1[ETHM] = ethm_update(P, W1, pos + 3 * (size_t)c);
  if (W1[ETHM] <= 0.0) W1[ETHM] = W0[ETHM];
  else W1[ENTR] = entropy_from_ethm(P, W1);
  const double idt = 1.0 / dt;
  R rt[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) rt[k] = R((W1[k] - W0[k]) * idt);
  store_n<R, NF>(Wrec + 50 * (size_t)c + 40, rt);
  // collect_reconstruction: rung = max(rung, get_rung(dt)), tend = t + dt(rung)
  int rf = rung[c];
  const int rb = get_rung(P, dt, min_rung);
  rf = rf < rb ? rb : rf;
  rung[c] = rf;
  tend[c] = t_global + get_dt(P, rf);
}

// One thread per cell; in partial steps a fixed grid strides over clist.
template <typename R>
__global__ void __launch_bounds__(128) k_pred_cell(int n, Params P, const Sched *__restrict__ S,
    const int *__restrict__ off, const int2 *__restrict__ lfj, const int2 *__restrict__ s12,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ U,
    const R *__restrict__ fcon, const unsigned char *__restrict__ fcode,
    int *__restrict__ rung, double *__restrict__ tend, R *__restrict__ Wrec, const int *__restrict__ perm,
    const int *__restrict__ clist) {
  const double t_global = S->t_global;
  const int min_rung = S->min_rung;
  const int cnt = clist ? S->ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x)
    pred_cell_body<R>(lst ? clist[t] : perm[t], t_global, min_rung, P, off, lfj, cvol, act, bnd, pos, U, fcon,
                      fcode, rung, tend, Wrec);
}

// ---- compute_reconstruction (MPI/compute_reconstruction.cpp:41-198) -------
// TPC threads per active cell, KH primitives each: Voronoi face gradient of
// the updated primitives, local limiter, density positivity rescale.
template <typename R, int KH>
__device__ __forceinline__ void recon_body(int c, int k0, const Params &P, const int *__restrict__ off,
    const int2 *__restrict__ lfj, const double *__restrict__ cvol, const unsigned char *__restrict__ act,
    const int *__restrict__ bnd, const R *__restrict__ Wst, const int *__restrict__ rung, R *__restrict__ Wrec,
    R *__restrict__ mnmx, unsigned char *__restrict__ mz, const R *__restrict__ lrw, const R *__restrict__ lrd,
    const unsigned char *__restrict__ bnb) {
  if (!(act[c] & A_ACTIVE)) return;
  R *r = Wrec + 50 * (size_t)c + k0;
  const R *wsi = Wst + 10 * (size_t)c + k0;
  R Wi[KH];
  load_n<R, KH>(wsi, Wi);
  if (bnd[c] != NO_BOUNDARY) {
#pragma unroll
    for (int k = 0; k < KH; k++) { r[k] = Wi[k]; r[10 + k] = R(0); r[20 + k] = R(0); r[30 + k] = R(0); r[40 + k] = R(0); }
    if (k0 == 0) mz[c] = 1;
    return;
  }
  const int q0 = off[c], q1 = off[c + 1];
  R Wx[KH], Wy[KH], Wz[KH], mn[KH], mx[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { Wx[k] = Wy[k] = Wz[k] = mn[k] = mx[k] = R(0); }
  // a boundary neighbour zeroes the reconstruction (its min/max are then unused)
  const bool zero = bnb[c] != 0;
  const int qe = zero ? q0 : q1;
  auto face_term = [&](const R *w6, const R *Wj) {
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R wj = Wj[k];
      const R sum = wj + Wi[k];
      const R diff = wj - Wi[k];
      mn[k] = smin(mn[k], diff);
      mx[k] = smax(mx[k], diff);
      Wx[k] += sum * w6[0] + diff * w6[3];
      Wy[k] += sum * w6[1] + diff * w6[4];
      Wz[k] += sum * w6[2] + diff * w6[5];
    }
  };
  FVM_CELL_LOOP
  for (int q = q0; q < qe; q++) {
    const int2 fj = lfj[q];
    const int j = fj.y >= 0 ? fj.y : ~fj.y;
    R w6[6];
    load_n<R, 6>(lrw + 6 * (size_t)q, w6);
    R Wj[KH];
    load_n<R, KH>(Wst + 10 * (size_t)j + k0, Wj);
    face_term(w6, Wj);
  }
  // the next step's limiter pass 1 (neighbour min/max of the same states)
  {
    R *mm = mnmx + 20 * (size_t)c + k0;
    { store_n<R, KH>(mm, mn); store_n<R, KH>(mm + 10, mx); }
    if (k0 == 0) mz[c] = zero ? 1 : 0;
  }
  if (zero) {
#pragma unroll
    for (int k = 0; k < KH; k++) { r[k] = Wi[k]; r[10 + k] = R(0); r[20 + k] = R(0); r[30 + k] = R(0); r[40 + k] = R(0); }
    return;
  }
  const R invV = R(1.0 / cvol[c]);
  R ln[KH], lq[KH], thr[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) {
    Wx[k] *= invV; Wy[k] *= invV; Wz[k] *= invV; ln[k] = R(2); lq[k] = R(1);
    thr[k] = limiter_thr(mn[k], mx[k]);
  }
  double sc[3] = {0.0, 0.0, 0.0};
  FVM_CELL_LOOP
  for (int q = q0; q < q1; q++) {
    const R *o3 = lrd + 3 * (size_t)q;
    const R dd[3] = {o3[0], o3[1], o3[2]};
    sc[0] = sc[0] + double(dd[0]); sc[1] = sc[1] + double(dd[1]); sc[2] = sc[2] + double(dd[2]);
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R dWx = Wx[k] * dd[0] + Wy[k] * dd[1] + Wz[k] * dd[2];
      limiter_ratio(ln[k], lq[k], dWx, mn[k], mx[k], thr[k]);
    }
  }
  R tt[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) {
    const R lm = limiter_finish(ln[k], lq[k]);
    Wx[k] *= lm; Wy[k] *= lm; Wz[k] *= lm;
    tt[k] = r[40 + k] * lm;
  }
  if (k0 == 0) {  // density positivity for the *-state (MPI/compute_reconstruction.cpp:179-197)
    const R sum_dt = R(get_dt(P, rung[c]));
    const R dWx = Wx[0] * R(sc[0]) + Wy[0] * R(sc[1]) + Wz[0] * R(sc[2]);
    const R dWp = dWx + tt[0] * sum_dt;
    const R dW = smax(dWx, dWp);
    if (dW > R(0)) {
      const R alpha = smin(R(1), R(0.9) * Wi[0] / dW);
      Wx[0] *= alpha; Wy[0] *= alpha; Wz[0] *= alpha; tt[0] *= alpha;
    }
  }
  store_n<R, KH>(r, Wi);
  store_n<R, KH>(r + 10, Wx);
  store_n<R, KH>(r + 20, Wy);
  store_n<R, KH>(r + 30, Wz);
  store_n<R, KH>(r + 40, tt);
}

// TPC threads per cell; in partial steps a fixed grid strides over clist.
template <typename R, int KH, int MINB>
__global__ void __launch_bounds__(128, MINB) k_recon(int n, Params P, const Sched *__restrict__ S,
    const int *__restrict__ off, const int2 *__restrict__ lfj,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const R *__restrict__ Wst, const int *__restrict__ rung, R *__restrict__ Wrec, const int *__restrict__ perm,
    R *__restrict__ mnmx, unsigned char *__restrict__ mz, const R *__restrict__ lrw,
    const R *__restrict__ lrd, const int *__restrict__ clist, const unsigned char *__restrict__ bnb) {
  constexpr int TPC = 10 / KH;
  const long long cnt = (long long)TPC * (clist ? S->ninv : n);
  const bool lst = clist && S->ninv != n;  // every cell involved: the list is the identity
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cnt;
       t += (long long)gridDim.x * blockDim.x) {
    const int u = (int)(t / TPC);
    recon_body<R, KH>(lst ? clist[u] : perm[u], (int)(t % TPC) * KH, P, off, lfj, cvol, act, bnd, Wst, rung, Wrec,
                      mnmx, mz, lrw, lrd, bnb);
  }
}

// Per link (a cell's entry in its face list, i.e. one side of a face), in the
// order the cell walks its faces: the face id and the neighbour j, stored as
// ~j when the cell is s2.  The mesh is fixed while it is installed.
// Cells with a boundary neighbour, whose reconstruction is zero (the
// reference's face loop stops at such a neighbour,
// MPI/compute_reconstruction.cpp:103-106,121); boundary codes are fixed
// after the state is installed.
__global__ void k_bnd_neighbours(int n, const int *__restrict__ off, const int2 *__restrict__ lfj,
                                 const int *__restrict__ bnd, unsigned char *__restrict__ bnb) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  unsigned char b = 0;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int2 fj = lfj[q];
    if (bnd[fj.y >= 0 ? fj.y : ~fj.y] != NO_BOUNDARY) b = 1;
  }
  bnb[c] = b;
}

__global__ void k_link_tables(int n, const int *__restrict__ off, const int *__restrict__ lnk,
                              const int2 *__restrict__ s12, int2 *__restrict__ lfj) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int f = lnk[q];
    const int2 e = s12[f];
    lfj[q] = make_int2(f, e.x == c ? e.y : ~e.x);
  }
}

__global__ void k_shared_sync(int n, Params P, const Sched *__restrict__ S, const unsigned char *__restrict__ act,
                              const int *__restrict__ iscal, int *__restrict__ rung, double *__restrict__ tend) {
  const double t_global = S->t_global;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(act[i] & A_ACTIVE)) return;
  const int r = iscal[0];
  rung[i] = r;
  tend[i] = t_global + get_dt(P, r);
}

// Scheduler::pull_active_list (MPI/Scheduler.h:108-154) on the device: the
// active rungs of this step are the set bits of tsysU ^ tnextU.
__global__ void k_sched_begin(Params P, Sched *S) {
  int max_rung = S->iscal[0];
  if (max_rung < 0 || max_rung >= RUNGMAX - 1) {
    S->iscal[2] |= 2;
    max_rung = max_rung < 0 ? 0 : RUNGMAX - 2;
  }
  const unsigned long long dtU = 1ULL << (RUNGMAX - 1 - max_rung);
  const unsigned long long tnextU = (S->tsysU / dtU + 1) * dtU;
  const unsigned long long flags = S->tsysU ^ tnextU;
  int min_rung = S->min_rung;
  for (int b = 0; b < RUNGMAX; b++)
    if (flags & (1ULL << b)) min_rung = RUNGMAX - 1 - b;
  S->max_rung = max_rung;
  S->min_rung = min_rung;
  S->flags = flags;
  S->tprevU = S->tsysU;
  S->tsysU = tnextU;
  S->t_global = P.dt_tick * (double)tnextU;
  S->dtmin = FVM_HUGE;
  S->iscal[0] = 0;
  S->iscal[1] = 0;
  S->iscal[3] = 0;
}

__global__ void k_sched_end(Sched *S, int n) {
  S->mnmx_ok = S->iscal[1] == n;
  S->nactive_total += (unsigned long long)S->iscal[1];
  S->nfaces_total += (unsigned long long)S->iscal[3];
  S->steps += 1;
}

__global__ void k_sched_set(Params P, Sched *S, unsigned long long tsysU, int reset_err) {
  S->tsysU = S->tprevU = tsysU;
  S->t_global = P.dt_tick * (double)tsysU;
  S->mnmx_ok = 0;  // the state was replaced
  if (reset_err) {
    S->min_rung = 0;
    S->iscal[2] = 0;
    S->nactive_total = S->nfaces_total = S->steps = 0;
  }
}

// Largest rung: a grid-stride maximum, one atomic per block.
__global__ void k_maxrung(int n, const int *__restrict__ rung, int *__restrict__ out) {
  int r = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r = max(r, rung[i]);
  for (int o = 16; o > 0; o >>= 1) r = max(r, __shfl_xor_sync(0xffffffffu, r, o));
  __shared__ int wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = max(r, wm[w]);
    atomicMax(out, r);
  }
}

// ---- init: compute_pvel + compute_timesteps(true) -------------------------
__global__ void k_init_dt(int n, Params P, const int *__restrict__ bnd, const double *__restrict__ U,
                          const double *__restrict__ volp, const double *__restrict__ vel,
                          const double *__restrict__ pos, double *__restrict__ dmin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double vmin = FVM_HUGE;
  if (i < n)
    vmin = smin(extra_timestep(P, i, bnd, pos, vel),
                cell_timestep(P, i, false, nullptr, nullptr, bnd, U, volp, vel));
  for (int o = 16; o > 0; o >>= 1) vmin = smin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0) atomic_min_pos(dmin, vmin);
}

template <typename R>
__global__ void k_init_state(int n, const double *__restrict__ W, const double *__restrict__ cvol,
                             double *__restrict__ U, double *__restrict__ dU, R *__restrict__ Wrec,
                             double *__restrict__ volp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double w[NF], u[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) w[k] = W[10 * (size_t)i + k];
  to_conservative(w, cvol[i], u);
#pragma unroll
  for (int k = 0; k < NF; k++) U[10 * (size_t)i + k] = u[k];
  for (int k = 0; k < 14; k++) dU[14 * (size_t)i + k] = 0.0;
  for (int k = 0; k < 50; k++) Wrec[50 * (size_t)i + k] = R(k < NF ? w[k] : 0.0);
  volp[i] = cvol[i];
}

template <typename R>
__global__ void k_limited_wrec(int n, const unsigned char *__restrict__ act, const R *__restrict__ Wrec,
                               const R *__restrict__ tau, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const R *r = Wrec + 50 * (size_t)i;
  double *o = out + 50 * (size_t)i;
  const bool imp = act[i] & (A_ACTIVE | A_LNGB);
  for (int k = 0; k < 50; k++) {
    const int v = k % 10;
    o[k] = double((k >= 10 && imp) ? r[k] * tau[10 * (size_t)i + v] : r[k]);
  }
}

template <typename A, typename B>
__global__ void k_convert(long long n, const A *__restrict__ in, B *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = B(in[i]);
}

__global__ void k_flux_kat(int nf, Params P, const double *wij, const double *Wi, const double *Wj,
                           const int *jbnd, const double *nrm, double *psi, double *Bn, double *flux) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double a[NF], b[NF], F[NF], w[3], nn[3], p, bn;
  for (int k = 0; k < NF; k++) { a[k] = Wi[10 * (size_t)f + k]; b[k] = Wj[10 * (size_t)f + k]; }
  for (int k = 0; k < 3; k++) { w[k] = wij[3 * (size_t)f + k]; nn[k] = nrm[3 * (size_t)f + k]; }
  compute_flux<double>(P, w, a, b, jbnd ? jbnd[f] : 0, nn, p, bn, F);
  psi[f] = p;
  Bn[f] = bn;
  for (int k = 0; k < NF; k++) flux[10 * (size_t)f + k] = F[k];
}

inline int nblk(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

// ============================== host context ================================

enum KernelId { KT_FLAGS = 0, KT_LIMITER, KT_CORR_FLUX, KT_CORR_CELL, KT_PVEL, KT_TIMESTEP, KT_RUNGS,
                KT_WST, KT_PRED_FLUX, KT_PRED_CELL, KT_RECON, KT_SYNC, KT_COUNT };
static const char *kKernelNames[KT_COUNT] = {"flags", "limiter", "corr_flux", "corr_cell", "pvel", "timestep",
                                             "rungs", "wst", "pred_flux", "pred_cell", "recon", "sync"};

// Per-device one-time settings (kernel attributes) are kept for device
// indices below this bound.
constexpr int kMaxDevices = 64;

struct fvm_ctx {
  int device;
  int sms = 148;  // SMs of the device (sizes the fixed grids of partial steps)
  // the flux passes walk the compacted active-face list (individual-timestep
  // steps and the stage-by-stage entry points) or every face (global steps)
  int use_flist = 1;
  // per-kernel CUDA-event timing (enabled by fvm_set_profiling)
  bool prof;
  cudaEvent_t kev[2 * KT_COUNT];
  bool kev_pending[KT_COUNT];
  double kt_ms[KT_COUNT];
  long long kt_calls[KT_COUNT];
  long long launches;
  cudaStream_t st;
  cudaEvent_t ev0, ev1;
  fvm_params prm;
  Params P;
  int n, nf;
  long long nl;
  // scheduler (MPI/Scheduler.h)
  unsigned long long tsysU;
  int min_rung, max_rung;
  double t_global;
  bool have_mesh, have_state, in_step;
  bool fp32;    // bulk (reconstruction, limiter, flux) in single precision
  size_t rb;    // bytes of one bulk value
  unsigned long long cur_flags;
  Dev d;
  std::vector<long long> h_off;
  std::vector<int> h_ids;
  bool keep_step_dU;
  float last_ms;
  // one captured step per mode (shared / individual), replayed by fvm_run
  cudaGraphExec_t graph[2];
  Sched hS;  // host copy of the device scheduler, refreshed after synchronisation
  // learned flux network: BF16 weight image and FP32 biases
  unsigned char *mlp_img = nullptr;
  float *mlp_bias = nullptr;
  int *mlp_err = nullptr;
  float *mlp_param = nullptr;  // FP32 master parameters
  // learned-flux mode: 0 exact, 1 network on gated faces, 2 exact + harvest
  int learn_mode = 0;
  LearnBuf lb{};
  float h_norm[48];  // standardisation of the network's inputs and outputs (fvm_mlp_set_norm)
  // launch choices of the autotuner (fvm_autotune); the defaults are the
  // tuned values of the 128^3 blast
  struct {
    int lim_staged = FVM_LIMITER_STAGE;  // staged limiter (shared-memory face records) or one record per thread
    int bs_face = 64;    // threads per block of the face kernels
    int bs_cell = 64;    // threads per block of the one-thread-per-cell gathers
    int bs_cell2 = 64;   // threads per block of the two-threads-per-cell kernels
  } tune;
  std::string err;
};

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);                        \
      return FVM_ECUDA;                                                                   \
    }                                                                                     \
  } while (0)

#define LAUNCH_CHECK()                                                                    \
  do {                                                                                    \
    c->launches++;                                                                        \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      c->err = std::string("kernel launch: ") + cudaGetErrorString(e_);                   \
      return FVM_ECUDA;                                                                   \
    }                                                                                     \
  } while (0)

static void kt_begin(fvm_ctx *c, int id) {
  if (c->prof) cudaEventRecord(c->kev[2 * id], c->st);
}
static void kt_end(fvm_ctx *c, int id) {
  if (c->prof) {
    cudaEventRecord(c->kev[2 * id + 1], c->st);
    c->kev_pending[id] = true;
  }
}
// called after a stream synchronisation: fold pending event pairs into totals
static void kt_collect(fvm_ctx *c) {
  if (!c->prof) return;
  for (int k = 0; k < KT_COUNT; k++)
    if (c->kev_pending[k]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->kev[2 * k], c->kev[2 * k + 1]) == cudaSuccess) {
        c->kt_ms[k] += ms;
        c->kt_calls[k]++;
      }
      c->kev_pending[k] = false;
    }
}

template <typename T>
static int dalloc(fvm_ctx *c, T **p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
  if (e != cudaSuccess) {
    c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return FVM_ENOMEM;
  }
  return 0;
}

static int dalloc_bytes(fvm_ctx *c, void **p, size_t bytes) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return FVM_ENOMEM;
  }
  return 0;
}

// Runs the statement with R bound to the context's bulk type.
#define BULK(...)                  \
  do {                             \
    if (c->fp32) {                 \
      using R = float;             \
      __VA_ARGS__;                 \
    } else {                       \
      using R = double;            \
      __VA_ARGS__;                 \
    }                              \
  } while (0)

// Grid of a kernel that strides over a device-side count of items (at most
// `items`): in partial steps (use_flist) a fixed grid of two full waves
// (4096 threads per SM), so a step with few active items launches few blocks
// and a step with many still fills every SM; otherwise one thread per item.
static int sgrid(const fvm_ctx *c, long long items, int bs) {
  const int g = nblk(items, bs);
  const int cap = c->sms * (4096 / bs);
  return (c->use_flist && g > cap) ? cap : g;
}

static void drop_graphs(fvm_ctx *c) {
  for (int k = 0; k < 2; k++)
    if (c->graph[k]) {
      cudaGraphExecDestroy(c->graph[k]);
      c->graph[k] = nullptr;
    }
}

static void free_all(fvm_ctx *c) {
  void **ptrs = (void **)&c->d;
  for (size_t k = 0; k < sizeof(Dev) / sizeof(void *); k++)
    if (ptrs[k]) cudaFree(ptrs[k]);
  memset(&c->d, 0, sizeof(Dev));
}

extern "C" {

fvm_ctx *fvm_create(const fvm_params *p, int device) {
  if (!p) return nullptr;
  fvm_ctx *c = new fvm_ctx();
  c->device = device;
  if (cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || c->sms <= 0)
    c->sms = 148;
  for (int k = 0; k < 48; k++)  // identity standardisation until fvm_mlp_set_norm
    c->h_norm[k] = (k < 16 || (k >= 32 && k < 40)) ? 0.0f : 1.0f;
  c->prm = *p;
  memset(&c->d, 0, sizeof(Dev));
  c->P.gamma = p->gamma;
  c->P.courant = p->courant;
  for (int a = 0; a < 3; a++) c->P.box[a] = p->box[a];
  c->P.dtmax = p->dtmax;
  c->P.dt_tick = p->dtmax / (double)(1ULL << (RUNGMAX - 1));
  c->P.eos = p->eos;
  c->P.iso_GM = p->iso_GM;
  c->P.iso_cfac = p->iso_cfac;
  c->P.static_mesh = p->static_mesh ? 1 : 0;
  c->tsysU = 0;
  c->min_rung = 0;
  c->max_rung = RUNGMAX - 1;
  c->t_global = 0.0;
  c->keep_step_dU = getenv("FVM_KEEP_STEP_DU") != nullptr;
  if (p->precision != FVM_PREC_FP64 && p->precision != FVM_PREC_FP32) { delete c; return nullptr; }
  c->fp32 = p->precision == FVM_PREC_FP32;
  c->rb = c->fp32 ? sizeof(float) : sizeof(double);
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return nullptr;
  }
  for (int k = 0; k < 2 * KT_COUNT; k++) cudaEventCreate(&c->kev[k]);
  return c;
}

void fvm_destroy(fvm_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  drop_graphs(c);
  free_all(c);
  if (c->mlp_img) cudaFree(c->mlp_img);
  if (c->mlp_bias) cudaFree(c->mlp_bias);
  if (c->mlp_err) cudaFree(c->mlp_err);
  if (c->mlp_param) cudaFree(c->mlp_param);
  for (int k = 0; k < 2 * KT_COUNT; k++) cudaEventDestroy(c->kev[k]);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaStreamDestroy(c->st);
  delete c;
}

const char *fvm_last_error(const fvm_ctx *c) { return c ? c->err.c_str() : "null context"; }

int fvm_set_mesh(fvm_ctx *c, int ncell, int nface, const int *s1, const int *s2, const double *n,
                 const double *centroid, const double *cell_volume, const double *cell_centroid,
                 const long long *off, const int *ids) {
  if (!c || ncell <= 0 || nface < 0 || !s1 || !s2 || !n || !centroid || !cell_volume || !cell_centroid || !off || !ids) {
    if (c) c->err = "fvm_set_mesh: bad argument";
    return FVM_EINVAL;
  }
  const long long nl = off[ncell];
  if (off[0] != 0 || nl < 0 || nl > 0x7fffffffLL) { c->err = "fvm_set_mesh: bad CSR offsets"; return FVM_EINVAL; }
  if (nface >= (1 << 28)) { c->err = "fvm_set_mesh: more than 2^28 faces"; return FVM_ERANGE; }
  for (int f = 0; f < nface; f++)
    if (s1[f] < 0 || s1[f] >= ncell || s2[f] < 0 || s2[f] >= ncell || s1[f] == s2[f]) {
      c->err = "fvm_set_mesh: face " + std::to_string(f) + " has a bad cell index";
      return FVM_EINVAL;
    }
  for (long long q = 0; q < nl; q++)
    if (ids[q] < 0 || ids[q] >= nface) { c->err = "fvm_set_mesh: bad face id in cell lists"; return FVM_EINVAL; }
  for (int i = 0; i < ncell; i++)
    if (off[i + 1] < off[i]) { c->err = "fvm_set_mesh: CSR offsets decrease"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  drop_graphs(c);
  free_all(c);
  c->learn_mode = 0;
  c->lb = LearnBuf{};
  c->n = ncell;
  c->nf = nface;
  c->nl = nl;
  int rc = 0;
  Dev &d = c->d;
  rc |= dalloc(c, &d.s12, nface); rc |= dalloc(c, &d.geo, nface); rc |= dalloc(c, &d.cen, nface);
  rc |= dalloc(c, &d.dr1, nface); rc |= dalloc(c, &d.dr2, nface); rc |= dalloc(c, &d.fflag, nface);
  rc |= dalloc_bytes(c, &d.fst, 20 * c->rb * (size_t)nface);
  rc |= dalloc(c, &d.cvol, ncell); rc |= dalloc(c, &d.ccen, 3 * (size_t)ncell);
  rc |= dalloc(c, &d.off, ncell + 1); rc |= dalloc(c, &d.lnk, nl); rc |= dalloc(c, &d.perm, ncell);
  rc |= dalloc(c, &d.lfj, nl);
  rc |= dalloc(c, &d.lsort, nl); rc |= dalloc(c, &d.lpart, nl);
  rc |= dalloc(c, &d.rdv, nl); rc |= dalloc(c, &d.wrv, nl); rc |= dalloc(c, &d.dt0, ncell);
  rc |= dalloc(c, &d.aflag, 8);
  rc |= dalloc(c, &d.awork, 2 * (size_t)ncell);
  rc |= dalloc_bytes(c, &d.mnmx, 20 * c->rb * (size_t)ncell); rc |= dalloc(c, &d.mz, ncell);
  rc |= dalloc_bytes(c, &d.lrw, 6 * c->rb * (size_t)nl);
  rc |= dalloc_bytes(c, &d.lrd, 3 * c->rb * (size_t)nl);
  rc |= dalloc_bytes(c, &d.lld, 3 * c->rb * (size_t)nl);
  rc |= dalloc(c, &d.alist, ncell); rc |= dalloc(c, &d.bcount, (ncell + CB - 1) / CB + 1);
  if ((ncell + CB - 1) / CB > CB * 16) { c->err = "fvm_set_mesh: more than 16M cells"; return FVM_ERANGE; }
  rc |= dalloc(c, &d.pos, 3 * (size_t)ncell); rc |= dalloc(c, &d.vel, 3 * (size_t)ncell);
  rc |= dalloc(c, &d.opos, 3 * (size_t)ncell); rc |= dalloc(c, &d.ovel, 3 * (size_t)ncell);
  rc |= dalloc(c, &d.divb, ncell);
  rc |= dalloc(c, &d.tlast, ncell); rc |= dalloc(c, &d.tend, ncell); rc |= dalloc(c, &d.volp, ncell);
  rc |= dalloc(c, &d.rung, ncell); rc |= dalloc(c, &d.bnd, ncell);
  rc |= dalloc(c, &d.U, 10 * (size_t)ncell); rc |= dalloc(c, &d.dU, 14 * (size_t)ncell);
  rc |= dalloc_bytes(c, &d.Wrec, 50 * c->rb * (size_t)ncell);
  rc |= dalloc(c, &d.act0, ncell); rc |= dalloc(c, &d.act, ncell); rc |= dalloc(c, &d.hash, ncell);
  rc |= dalloc(c, &d.fcode, nface); rc |= dalloc(c, &d.fcode2, nface);
  rc |= dalloc(c, &d.flist, nface); rc |= dalloc(c, &d.fbcount, (nface + CB - 1) / CB + 1);
  rc |= dalloc(c, &d.clist, ncell); rc |= dalloc(c, &d.cbcount, (ncell + CB - 1) / CB + 1);
  rc |= dalloc(c, &d.bnb, ncell);
  rc |= dalloc_bytes(c, &d.tau, 10 * c->rb * (size_t)ncell);
  rc |= dalloc_bytes(c, &d.fcon, 14 * c->rb * (size_t)nface);
  rc |= dalloc_bytes(c, &d.fcon2, 14 * c->rb * (size_t)nface);
  rc |= dalloc_bytes(c, &d.Wst, 10 * c->rb * (size_t)ncell);
  rc |= dalloc(c, &d.dtl, ncell);
  if (c->keep_step_dU) rc |= dalloc(c, &d.stepdU, 14 * (size_t)ncell);
  rc |= dalloc(c, &d.S, 1); rc |= dalloc(c, &d.counters, 4);
  if (rc) return FVM_ENOMEM;
  // no face active yet, every face coded F_OFF (k_faceflags keeps this so for
  // the faces it turns inactive)
  CK(cudaMemsetAsync(d.fflag, 0, nface, c->st));
  CK(cudaMemsetAsync(d.fcode, F_OFF, nface, c->st));
  CK(cudaMemsetAsync(d.fcode2, F_OFF, nface, c->st));
  std::vector<int2> hs(nface);
  std::vector<double4> hg(nface), hc(nface);
  for (int f = 0; f < nface; f++) {
    hs[f] = make_int2(s1[f], s2[f]);
    const double *v = n + 3 * (size_t)f;
    const double area = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double ia = 1.0 / area;
    hg[f] = make_double4(v[0] * ia, v[1] * ia, v[2] * ia, area);
    const double *q = centroid + 3 * (size_t)f;
    hc[f] = make_double4(q[0], q[1], q[2], 0.0);
  }
  std::vector<int> hoff(ncell + 1);
  for (int i = 0; i <= ncell; i++) hoff[i] = (int)off[i];
  c->h_off.assign(off, off + ncell + 1);
  c->h_ids.assign(ids, ids + nl);
  CK(cudaMemcpy(d.s12, hs.data(), sizeof(int2) * nface, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.geo, hg.data(), sizeof(double4) * nface, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.cen, hc.data(), sizeof(double4) * nface, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.cvol, cell_volume, sizeof(double) * ncell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.ccen, cell_centroid, sizeof(double) * 3 * ncell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.off, hoff.data(), sizeof(int) * (ncell + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.lnk, ids, sizeof(int) * nl, cudaMemcpyHostToDevice));
  {
    // every face must be listed once by each of its two cells: the link of
    // the other side, and each cell's links ordered by neighbour index
    std::vector<int> flink(2 * (size_t)nface, -1), part(nl), srt(nl);
    for (int c0 = 0; c0 < ncell; c0++)
      for (long long q = off[c0]; q < off[c0 + 1]; q++) {
        const int f = ids[q];
        const int side = s1[f] == c0 ? 0 : (s2[f] == c0 ? 1 : -1);
        if (side < 0 || flink[2 * (size_t)f + side] >= 0) {
          c->err = "fvm_set_mesh: face " + std::to_string(f) + " listed by a cell that is not its side, or twice";
          return FVM_EINVAL;
        }
        flink[2 * (size_t)f + side] = (int)q;
      }
    for (int f = 0; f < nface; f++) {
      const int a = flink[2 * (size_t)f], b = flink[2 * (size_t)f + 1];
      if (a < 0 || b < 0) {
        c->err = "fvm_set_mesh: face " + std::to_string(f) + " missing from a cell's face list";
        return FVM_EINVAL;
      }
      part[a] = b;
      part[b] = a;
    }
    for (int c0 = 0; c0 < ncell; c0++) {
      const long long q0 = off[c0], q1 = off[c0 + 1];
      for (long long q = q0; q < q1; q++) srt[q] = (int)q;
      auto nb = [&](int q) { const int f = ids[q]; return s1[f] == c0 ? s2[f] : s1[f]; };
      std::sort(srt.begin() + q0, srt.begin() + q1, [&](int x, int y) { return nb(x) < nb(y); });
    }
    CK(cudaMemcpy(d.lpart, part.data(), sizeof(int) * nl, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.lsort, srt.data(), sizeof(int) * nl, cudaMemcpyHostToDevice));
    k_link_tables<<<nblk(ncell, 256), 256, 0, c->st>>>(ncell, d.off, d.lnk, d.s12, d.lfj);
    LAUNCH_CHECK();
    CK(cudaStreamSynchronize(c->st));
  }
  {
    std::vector<int> perm(ncell);
    for (int i = 0; i < ncell; i++) perm[i] = i;
#if FVM_CELL_PERM
    for (int w0 = 0; w0 < ncell; w0 += CPW) {
      const int w1 = std::min(ncell, w0 + CPW);
      std::stable_sort(perm.begin() + w0, perm.begin() + w1,
                       [&](int a, int b) { return off[a + 1] - off[a] < off[b + 1] - off[b]; });
    }
#endif
    CK(cudaMemcpy(d.perm, perm.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice));
  }
  CK(cudaMemsetAsync(d.counters, 0, 4 * sizeof(unsigned long long), c->st));
  CK(cudaStreamSynchronize(c->st));
  c->have_mesh = true;
  c->have_state = false;
  return 0;
}

// Synchronise and refresh the host copy of the scheduler.
static int read_sched(fvm_ctx *c) {
  CK(cudaMemcpyAsync(&c->hS, c->d.S, sizeof(Sched), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->tsysU = c->hS.tsysU;
  c->t_global = c->hS.t_global;
  c->min_rung = c->hS.min_rung;
  c->max_rung = c->hS.max_rung;
  return 0;
}

// Rung maximum over all cells into S->iscal[0] (the next step's max_rung).
static int enqueue_maxrung(fvm_ctx *c) {
  CK(cudaMemsetAsync(&c->d.S->iscal[0], 0, sizeof(int), c->st));
  k_maxrung<<<smin(nblk(c->n, 256), 4 * c->sms), 256, 0, c->st>>>(c->n, c->d.rung, &c->d.S->iscal[0]);
  LAUNCH_CHECK();
  return 0;
}

int fvm_init_problem(fvm_ctx *c, const double *W, const double *pos, const int *bnd, int rung_offset) {
  if (!c || !W || !pos) { if (c) c->err = "fvm_init_problem: bad argument"; return FVM_EINVAL; }
  if (!c->have_mesh) { c->err = "fvm_init_problem: no mesh"; return FVM_ENOMESH; }
  CK(cudaSetDevice(c->device));
  const int n = c->n;
  Dev &d = c->d;
  double *dW = nullptr;
  CK(cudaMalloc(&dW, sizeof(double) * 10 * (size_t)n));
  cudaError_t e = cudaMemcpyAsync(dW, W, sizeof(double) * 10 * (size_t)n, cudaMemcpyHostToDevice, c->st);
  if (e != cudaSuccess) { cudaFree(dW); c->err = cudaGetErrorString(e); return FVM_ECUDA; }
  CK(cudaMemcpyAsync(d.pos, pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, c->st));
  if (bnd) CK(cudaMemcpyAsync(d.bnd, bnd, sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
  else CK(cudaMemsetAsync(d.bnd, 0, sizeof(int) * n, c->st));
  k_bnd_neighbours<<<nblk(n, 256), 256, 0, c->st>>>(n, d.off, d.lfj, d.bnd, d.bnb);
  LAUNCH_CHECK();
  CK(cudaMemsetAsync(d.vel, 0, sizeof(double) * 3 * (size_t)n, c->st));
  CK(cudaMemsetAsync(d.tlast, 0, sizeof(double) * n, c->st));
  k_face_geom<<<nblk(c->nf, 256), 256, 0, c->st>>>(c->nf, c->P, d.s12, d.geo, d.cen, d.pos, d.dr1, d.dr2);
  LAUNCH_CHECK();
  BULK(k_link_recon<R><<<nblk(n, 256), 256, 0, c->st>>>(n, c->P, d.off, d.lfj, d.geo, d.dr1, d.dr2, (R *)d.lrw,
                                                        (R *)d.lrd, (R *)d.lld));
  LAUNCH_CHECK();

  BULK(k_init_state<R><<<nblk(n, 128), 128, 0, c->st>>>(n, dW, d.cvol, d.U, d.dU, (R *)d.Wrec, d.volp));
  LAUNCH_CHECK();
  // compute_pvel on all cells, then the shared timestep
  CK(cudaMemsetAsync(d.act, A_ACTIVE, n, c->st));
  k_pvel<<<nblk(n, 128), 128, 0, c->st>>>(n, c->P, d.act, d.bnd, d.U, d.volp, d.cvol, d.ccen, d.pos, d.vel, nullptr,
                                          nullptr);
  LAUNCH_CHECK();
  CK(cudaMemcpyAsync(d.opos, d.pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemcpyAsync(d.ovel, d.vel, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemsetAsync(d.divb, 0, sizeof(float) * n, c->st));
  Sched h0;
  memset(&h0, 0, sizeof(h0));
  h0.dtmin = FVM_HUGE;
  CK(cudaMemcpyAsync(d.S, &h0, sizeof(Sched), cudaMemcpyHostToDevice, c->st));
  k_init_dt<<<nblk(n, 128), 128, 0, c->st>>>(n, c->P, d.bnd, d.U, d.volp, d.vel, d.pos, &d.S->dtmin);
  LAUNCH_CHECK();
  double dtmin = 0.0;
  CK(cudaMemcpyAsync(&dtmin, &d.S->dtmin, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  cudaFree(dW);
  c->min_rung = 0;
  const int rung = get_rung(c->P, dtmin, c->min_rung) + rung_offset;
  if (rung < 0 || rung >= RUNGMAX - 1) { c->err = "fvm_init_problem: initial rung out of range"; return FVM_ERANGE; }
  std::vector<int> hr(n, rung);
  std::vector<double> ht(n, 0.0 + get_dt(c->P, rung));
  CK(cudaMemcpy(d.rung, hr.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.tend, ht.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  h0.iscal[0] = rung;  // max rung for the first pull
  CK(cudaMemcpyAsync(d.S, &h0, sizeof(Sched), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->tsysU = 0;
  c->t_global = 0.0;
  c->max_rung = rung;
  c->min_rung = 0;
  c->have_state = true;
  c->in_step = false;
  drop_graphs(c);
  return 0;
}

int fvm_get_state(fvm_ctx *c, double *pos, double *vel, double *tlast, double *tend, int *rung, double *U,
                  double *dU, double *wrec) {
  if (!c || !c->have_mesh) return FVM_ENOMESH;
  CK(cudaSetDevice(c->device));
  const size_t n = c->n;
  cudaStream_t s = c->st;
  if (pos) CK(cudaMemcpyAsync(pos, c->d.pos, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (vel) CK(cudaMemcpyAsync(vel, c->d.vel, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (tlast) CK(cudaMemcpyAsync(tlast, c->d.tlast, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (tend) CK(cudaMemcpyAsync(tend, c->d.tend, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (rung) CK(cudaMemcpyAsync(rung, c->d.rung, n * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (U) CK(cudaMemcpyAsync(U, c->d.U, 10 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (dU) CK(cudaMemcpyAsync(dU, c->d.dU, 14 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (wrec && !c->fp32) CK(cudaMemcpyAsync(wrec, c->d.Wrec, 50 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (wrec && c->fp32) {
    double *tmp = nullptr;
    CK(cudaMallocAsync(&tmp, 50 * n * sizeof(double), s));
    k_convert<float, double><<<nblk(50LL * n, 256), 256, 0, s>>>(50LL * n, (const float *)c->d.Wrec, tmp);
    CK(cudaMemcpyAsync(wrec, tmp, 50 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(tmp, s));
  }
  CK(cudaStreamSynchronize(s));
  return 0;
}

int fvm_set_state(fvm_ctx *c, const double *vel, const double *tlast, const double *tend, const int *rung,
                  const double *U, const double *dU, const double *wrec, unsigned long long tsys_ticks) {
  if (!c || !c->have_mesh) return FVM_ENOMESH;
  if (c->in_step) { c->err = "fvm_set_state: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const size_t n = c->n;
  cudaStream_t s = c->st;
  if (rung) {
    for (size_t i = 0; i < n; i++)
      if (rung[i] < 0 || rung[i] >= RUNGMAX - 1) { c->err = "fvm_set_state: rung out of range"; return FVM_ERANGE; }
    CK(cudaMemcpyAsync(c->d.rung, rung, n * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  if (vel) CK(cudaMemcpyAsync(c->d.vel, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (tlast) CK(cudaMemcpyAsync(c->d.tlast, tlast, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (tend) CK(cudaMemcpyAsync(c->d.tend, tend, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (U) CK(cudaMemcpyAsync(c->d.U, U, 10 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (dU) CK(cudaMemcpyAsync(c->d.dU, dU, 14 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (wrec && !c->fp32) CK(cudaMemcpyAsync(c->d.Wrec, wrec, 50 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (wrec && c->fp32) {
    double *tmp = nullptr;
    CK(cudaMallocAsync(&tmp, 50 * n * sizeof(double), s));
    CK(cudaMemcpyAsync(tmp, wrec, 50 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    k_convert<double, float><<<nblk(50LL * n, 256), 256, 0, s>>>(50LL * n, tmp, (float *)c->d.Wrec);
    CK(cudaFreeAsync(tmp, s));
  }
  CK(cudaMemcpyAsync(c->d.volp, c->d.cvol, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  k_sched_set<<<1, 1, 0, s>>>(c->P, c->d.S, tsys_ticks, 0);
  LAUNCH_CHECK();
  int rc = enqueue_maxrung(c);
  if (rc) return rc;
  c->have_state = true;
  rc = read_sched(c);
  c->max_rung = c->hS.iscal[0];
  return rc;
}

// ---- step launches (no host synchronisation) ------------------------------

static int enq_begin(fvm_ctx *c) {
  const int n = c->n;
  Dev &d = c->d;
  kt_begin(c, KT_FLAGS);
  k_sched_begin<<<1, 1, 0, c->st>>>(c->P, d.S);
  LAUNCH_CHECK();
  k_active<<<nblk(n, 256), 256, 0, c->st>>>(n, d.rung, d.S, d.act, &d.S->iscal[1]);
  LAUNCH_CHECK();
  // partial steps: blocks of CB faces, whose counts start the face compaction
  k_faceflags<<<nblk(c->nf, CB), CB, 0, c->st>>>(c->nf, d.s12, d.act, d.bnd, d.fflag, &d.S->iscal[3], d.fcode,
                                                 d.fcode2, c->use_flist ? d.fbcount : nullptr);
  LAUNCH_CHECK();
  if (c->use_flist) {
    const int nb = (int)((c->nf + CB - 1) / CB);
    k_scan_counts<<<1, CB, 0, c->st>>>(nb, d.fbcount, &d.fbcount[nb]);
    LAUNCH_CHECK();
    k_place_faces<<<nb, CB, 0, c->st>>>(c->nf, d.fflag, &d.S->iscal[3], d.fbcount, d.flist);
    LAUNCH_CHECK();
    const int nbc = (int)((c->n + CB - 1) / CB);
    k_count_cells<<<nbc, CB, 0, c->st>>>(c->n, d.act, d.cbcount);
    LAUNCH_CHECK();
    k_scan_counts<<<1, CB, 0, c->st>>>(nbc, d.cbcount, &d.S->ninv);
    LAUNCH_CHECK();
    k_place_cells<<<nbc, CB, 0, c->st>>>(c->n, d.act, d.cbcount, d.clist);
    LAUNCH_CHECK();
  }
  kt_end(c, KT_FLAGS);
  return 0;
}

static int enq_limiter(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_LIMITER);
  static_assert(FVM_CELL_PERM == 0, "the staged limiter maps threads to consecutive cells");
  // Global steps: the staged limiter when the autotuner picked it, else the
  // per-thread one.  Partial steps launch both: the staged one (one block per
  // CST cells) works only in a step where every cell is active, the list one
  // (on a fixed grid) only in the others.
  const bool staged = c->tune.lim_staged != 0;
  if (staged) {
    BULK(({
      // the attribute is per device: set once on each device a context uses
      static bool attr[kMaxDevices] = {};
      if (c->device < 0 || c->device >= kMaxDevices) { c->err = "device index out of range"; return FVM_EINVAL; }
      if (!attr[c->device]) {
        CK(cudaFuncSetAttribute(k_limiter_st<R, CellTune<R>::KH_LIM, CellTune<R>::MINB_LIM>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                limiter_stage_bytes<R, CellTune<R>::KH_LIM>()));
        attr[c->device] = true;
      }
      k_limiter_st<R, CellTune<R>::KH_LIM, CellTune<R>::MINB_LIM>
          <<<nblk(c->n, limiter_cst<CellTune<R>::KH_LIM>()), 128,
             limiter_stage_bytes<R, CellTune<R>::KH_LIM>(), c->st>>>(
          c->n, c->P, d.S, d.off, d.lnk, d.lfj, d.s12, d.geo, d.dr1, d.fflag, d.act, d.tlast, (const R *)d.Wrec,
          (R *)d.tau, (R *)d.fst, d.perm, (const R *)d.mnmx, d.mz, c->use_flist, (const R *)d.lld);
    }));
    LAUNCH_CHECK();
  }
  if (!staged || c->use_flist) {
    const int bs = c->tune.bs_cell2;
    BULK(k_limiter<R, CellTune<R>::KH_LIM, CellTune<R>::MINB_LIM>
         <<<sgrid(c, (long long)(10 / CellTune<R>::KH_LIM) * c->n, bs), bs, 0, c->st>>>(c->n, c->P, d.S, d.off, d.lnk, d.lfj, d.s12, d.geo,
                                                              d.dr1, d.fflag, d.act, d.tlast, (const R *)d.Wrec,
                                                              (R *)d.tau, (R *)d.fst, d.perm, (const R *)d.mnmx,
                                                              d.mz, c->use_flist ? d.clist : nullptr,
                                                              staged && c->use_flist, (const R *)d.lld));
  }
  LAUNCH_CHECK();
  kt_end(c, KT_LIMITER);
  return 0;
}

static int mlp_launch_dev(fvm_ctx *c, int nmax, const int *n_dev, const __nv_bfloat16 *X, float *Y);

static int enq_update(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_CORR_FLUX);
  const LearnBuf &lb = c->lb;
#define CORR_FLUX(MODE, GRID)                                                                                   \
  BULK(k_corr_flux<R, MODE><<<GRID, c->tune.bs_face, 0, c->st>>>(c->nf, c->P, d.S, d.s12, d.geo, d.dr1, d.fflag, d.bnd, d.vel, \
                                                     d.tlast, (const R *)d.Wrec, (const R *)d.fst, (R *)d.fcon,   \
                                                     d.fcode, lb, d.flist, c->use_flist))
  if (c->learn_mode == 1) {
    CK(cudaMemsetAsync(lb.count, 0, sizeof(int), c->st));
    CORR_FLUX(LM_DEFER, sgrid(c, c->nf, c->tune.bs_face));
    LAUNCH_CHECK();
    int rc = mlp_launch_dev(c, c->nf, lb.count, lb.X, lb.Y);
    if (rc) return rc;
    CORR_FLUX(LM_FINISH, nblk(c->nf, c->tune.bs_face));
  } else if (c->learn_mode == 2) {
    CORR_FLUX(LM_HARVEST, sgrid(c, c->nf, c->tune.bs_face));
  } else {
    CORR_FLUX(LM_EXACT, sgrid(c, c->nf, c->tune.bs_face));
  }
#undef CORR_FLUX
  LAUNCH_CHECK();
  kt_end(c, KT_CORR_FLUX);
  kt_begin(c, KT_CORR_CELL);
  BULK(k_corr_cell<R><<<sgrid(c, c->n, c->tune.bs_cell), c->tune.bs_cell, 0, c->st>>>(c->n, c->P, d.S, d.off, d.lfj, d.s12, d.cvol, d.act,
                                                          d.bnd, d.pos, d.tlast, d.volp, (const R *)d.Wrec,
                                                          (const R *)d.tau, (const R *)d.fcon, d.fcode, d.U, d.dU,
                                                          d.stepdU, d.counters, d.perm, d.divb,
                                                          c->use_flist ? d.clist : nullptr));
  LAUNCH_CHECK();
  kt_end(c, KT_CORR_CELL);
  return 0;
}

static int enq_pvel(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_PVEL);
  k_pvel<<<sgrid(c, c->n, 128), 128, 0, c->st>>>(c->n, c->P, d.act, d.bnd, d.U, d.volp, d.cvol, d.ccen, d.pos, d.vel,
                                                 c->use_flist ? d.clist : nullptr, &d.S->ninv);
  LAUNCH_CHECK();
  kt_end(c, KT_PVEL);
  return 0;
}

static int enq_timesteps(fvm_ctx *c, int shared) {
  Dev &d = c->d;
  const int n = c->n;
  kt_begin(c, KT_TIMESTEP);
  const int *cl = c->use_flist ? d.clist : nullptr;  // partial steps: the involved cells only
  k_timestep<<<sgrid(c, n, 128), 128, 0, c->st>>>(n, c->P, d.off, d.lfj, d.act, d.bnd, d.U, d.volp, d.vel,
                                                  d.pos, d.tlast, d.tend, d.dtl, &d.S->dtmin, cl, &d.S->ninv);
  LAUNCH_CHECK();
  if (!shared) {
    k_halve<<<sgrid(c, n, 256), 256, 0, c->st>>>(n, d.act, &d.S->dtmin, d.dtl, cl, &d.S->ninv);
    LAUNCH_CHECK();
    CK(cudaMemsetAsync(d.hash, 0, n, c->st));
    CK(cudaMemsetAsync(&d.S->iscal[4], 0, 4 * sizeof(int), c->st));
    CK(cudaMemsetAsync(d.awork, 0, 2 * (size_t)n, c->st));
    CK(cudaMemsetAsync(d.act0, 0, n, c->st));
    k_adjust_mark<<<sgrid(c, n, 128), 128, 0, c->st>>>(n, d.off, d.lfj, d.act, d.bnd, d.dtl, d.hash,
                                                      &d.S->iscal[4], d.act0, d.awork, cl, &d.S->ninv);
    LAUNCH_CHECK();
    const int nb = (int)((n + CB - 1) / CB);
    k_count_flags<<<nb, CB, 0, c->st>>>(n, d.act0, d.bcount);
    LAUNCH_CHECK();
    k_scan_counts<<<1, CB, 0, c->st>>>(nb, d.bcount, &d.S->iscal[5]);
    LAUNCH_CHECK();
    k_place_flags<<<nb, CB, 0, c->st>>>(n, d.act0, d.bcount, d.alist);
    LAUNCH_CHECK();
#if FVM_ADJUST_REPLAY
    CK(cudaMemsetAsync(d.aflag, 0, 8 * sizeof(int), c->st));
    k_adjust_init<<<sgrid(c, n, 256), 256, 0, c->st>>>(n, d.off, d.lfj, d.act, &d.S->iscal[4], d.dtl, d.dt0,
                                                      d.rdv, d.wrv, d.aflag, cl, &d.S->ninv);
    LAUNCH_CHECK();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(c->st, &cs));
    const int rgrid = smin(nblk(n, 128), 16 * c->sms);
    if (cs == cudaStreamCaptureStatusActive) {
      // a WHILE node whose body is one replay and k_adjust_next: the step
      // graph runs as many replays as the relaxation needs, no launches after
      cudaGraph_t g;
      const cudaGraphNode_t *deps = nullptr;
      size_t nd = 0;
      CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
      cudaGraphConditionalHandle h;
      CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t cn;
      CK(cudaGraphAddNode(&cn, g, deps, nd, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      int k0 = 0, kdev = 1;
      void *ra[] = {(void *)&n, &k0, &d.off, &d.lfj, &d.lsort, &d.lpart, &d.act, &d.dt0, &d.rdv, &d.wrv, &d.dtl,
                    &d.aflag, &d.awork, &kdev};
      cudaKernelNodeParams kp = {};
      kp.func = (void *)k_adjust_replay;
      kp.gridDim = dim3(rgrid);
      kp.blockDim = dim3(128);
      kp.kernelParams = ra;
      cudaGraphNode_t kr, kx;
      CK(cudaGraphAddKernelNode(&kr, body, nullptr, 0, &kp));
      void *na[] = {&d.aflag, &h};
      cudaKernelNodeParams kn = {};
      kn.func = (void *)k_adjust_next;
      kn.gridDim = dim3(1);
      kn.blockDim = dim3(1);
      kn.kernelParams = na;
      CK(cudaGraphAddKernelNode(&kx, body, &kr, 1, &kn));
      CK(cudaStreamUpdateCaptureDependencies(c->st, &cn, 1, cudaStreamSetCaptureDependencies));
      c->launches += 2;
    } else {
      for (int k = 0; k < ADJ_ITERS; k++) {
        k_adjust_replay<<<rgrid, 128, 0, c->st>>>(n, k, d.off, d.lfj, d.lsort, d.lpart, d.act, d.dt0, d.rdv, d.wrv,
                                                  d.dtl, d.aflag, d.awork, 0);
        LAUNCH_CHECK();
      }
    }
    k_adjust_restore<<<sgrid(c, n, 256), 256, 0, c->st>>>(n, d.act, d.dt0, d.dtl, d.aflag, &d.S->iscal[6], cl,
                                                         &d.S->ninv);
    LAUNCH_CHECK();
    k_adjust_seq<<<1, 32, 0, c->st>>>(d.off, d.lnk, d.s12, d.alist, &d.S->iscal[5], &d.aflag[4], d.dtl);
#else
    k_adjust_seq<<<1, 32, 0, c->st>>>(d.off, d.lnk, d.s12, d.alist, &d.S->iscal[5], &d.S->iscal[4], d.dtl);
#endif
    LAUNCH_CHECK();
  }
  kt_end(c, KT_TIMESTEP);
  kt_begin(c, KT_RUNGS);
  BULK(k_rungs<R><<<sgrid(c, n, 256), 256, 0, c->st>>>(n, c->P, d.S, shared, d.act, d.hash, d.dtl, &d.S->dtmin, d.rung,
                                                   d.tlast, d.tend, (R *)d.Wrec, d.S->iscal, d.vel, d.opos,
                                                   d.ovel, c->use_flist ? d.clist : nullptr));
  LAUNCH_CHECK();
  kt_end(c, KT_RUNGS);
  return 0;
}

static int enq_collect(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_WST);
  BULK(k_wst<R><<<sgrid(c, c->n, 256), 256, 0, c->st>>>(c->n, d.act, d.U, d.volp, (R *)d.Wst,
                                                        c->use_flist ? d.clist : nullptr, &d.S->ninv));
  LAUNCH_CHECK();
  kt_end(c, KT_WST);
  return 0;
}

static int enq_update0(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_PRED_FLUX);
  const LearnBuf &lb = c->lb;
#define PRED_FLUX(MODE, GRID)                                                                                 \
  BULK(k_pred_flux<R, MODE><<<GRID, c->tune.bs_face, 0, c->st>>>(c->nf, c->P, d.s12, d.geo, d.dr1, d.fflag, d.bnd, \
                                                                 d.vel, (const R *)d.Wst, (R *)d.fcon2, d.fcode2, \
                                                                 d.S, d.rung, lb, d.flist, c->use_flist))
  if (c->learn_mode == 1) {
    CK(cudaMemsetAsync(lb.count, 0, sizeof(int), c->st));
    PRED_FLUX(LM_DEFER, sgrid(c, c->nf, c->tune.bs_face));
    LAUNCH_CHECK();
    int rc = mlp_launch_dev(c, c->nf, lb.count, lb.X, lb.Y);
    if (rc) return rc;
    PRED_FLUX(LM_FINISH, nblk(c->nf, c->tune.bs_face));
  } else if (c->learn_mode == 2) {
    PRED_FLUX(LM_HARVEST, sgrid(c, c->nf, c->tune.bs_face));
  } else {
    PRED_FLUX(LM_EXACT, sgrid(c, c->nf, c->tune.bs_face));
  }
#undef PRED_FLUX
  LAUNCH_CHECK();
  kt_end(c, KT_PRED_FLUX);
  return 0;
}

static int enq_recon(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_PRED_CELL);
  BULK(k_pred_cell<R><<<sgrid(c, c->n, c->tune.bs_cell), c->tune.bs_cell, 0, c->st>>>(c->n, c->P, d.S, d.off, d.lfj, d.s12, d.cvol, d.act,
                                                          d.bnd, d.pos, d.U, (const R *)d.fcon2, d.fcode2, d.rung,
                                                          d.tend, (R *)d.Wrec, d.perm, c->use_flist ? d.clist : nullptr));
  LAUNCH_CHECK();
  kt_end(c, KT_PRED_CELL);
  kt_begin(c, KT_RECON);
  BULK(k_recon<R, CellTune<R>::KH_REC, CellTune<R>::MINB_REC>
       <<<sgrid(c, (long long)(10 / CellTune<R>::KH_REC) * c->n, c->tune.bs_cell2), c->tune.bs_cell2, 0, c->st>>>(
           c->n, c->P, d.S, d.off, d.lfj, d.cvol, d.act, d.bnd, (const R *)d.Wst, d.rung, (R *)d.Wrec, d.perm,
           (R *)d.mnmx, d.mz, (const R *)d.lrw, (const R *)d.lrd, c->use_flist ? d.clist : nullptr, d.bnb));
  LAUNCH_CHECK();
  kt_end(c, KT_RECON);
  return 0;
}

static int enq_end(fvm_ctx *c, int shared) {
  Dev &d = c->d;
  kt_begin(c, KT_SYNC);
  int rc = enqueue_maxrung(c);
  if (rc) return rc;
  if (shared) {
    k_shared_sync<<<nblk(c->n, 256), 256, 0, c->st>>>(c->n, c->P, d.S, d.act, d.S->iscal, d.rung, d.tend);
    LAUNCH_CHECK();
  }
  k_sched_end<<<1, 1, 0, c->st>>>(d.S, c->n);
  LAUNCH_CHECK();
  kt_end(c, KT_SYNC);
  return 0;
}

static int enq_step(fvm_ctx *c, int shared) {
  int rc;
  c->use_flist = shared ? 0 : 1;  // a global step activates every face
  if ((rc = enq_begin(c))) return rc;
  if ((rc = enq_limiter(c))) return rc;
  if ((rc = enq_update(c))) return rc;
  if ((rc = enq_pvel(c))) return rc;
  if ((rc = enq_timesteps(c, shared))) return rc;
  if ((rc = enq_collect(c))) return rc;
  if ((rc = enq_update0(c))) return rc;
  if ((rc = enq_recon(c))) return rc;
  return enq_end(c, shared);
}

static int check_sched_errors(fvm_ctx *c) {
  if (c->hS.iscal[2]) {
    c->err = "rung left [0, 31) (flags " + std::to_string(c->hS.iscal[2]) + ")";
    return FVM_ERANGE;
  }
  return 0;
}

// ---- the reference call sequence, one entry point per member function -----

#define STEP_GUARD(name)                                                                  \
  do {                                                                                    \
    if (!c || !c->in_step) {                                                              \
      if (c) c->err = std::string(name) + ": call fvm_begin_step first";                  \
      return FVM_EINVAL;                                                                  \
    }                                                                                     \
  } while (0)

int fvm_begin_step(fvm_ctx *c) {
  if (!c || !c->have_state) { if (c) c->err = "fvm_begin_step: no state"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_begin_step: previous step not finished"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  c->use_flist = 1;
  int rc = enq_begin(c);
  if (rc) return rc;
  if ((rc = read_sched(c))) return rc;
  if ((rc = check_sched_errors(c))) return rc;
  c->in_step = true;
  return c->hS.iscal[1];
}

int fvm_slope_limiter(fvm_ctx *c) { STEP_GUARD("fvm_slope_limiter"); return enq_limiter(c); }
int fvm_compute_update(fvm_ctx *c) { STEP_GUARD("fvm_compute_update"); return enq_update(c); }
int fvm_compute_pvel(fvm_ctx *c) { STEP_GUARD("fvm_compute_pvel"); return enq_pvel(c); }

int fvm_compute_timesteps(fvm_ctx *c, int shared, double *dt_min_out) {
  STEP_GUARD("fvm_compute_timesteps");
  int rc = enq_timesteps(c, shared);
  if (rc) return rc;
  if (dt_min_out) {
    CK(cudaMemcpyAsync(dt_min_out, &c->d.S->dtmin, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return 0;
}

int fvm_collect_results(fvm_ctx *c) { STEP_GUARD("fvm_collect_results"); return enq_collect(c); }
int fvm_compute_update0(fvm_ctx *c) { STEP_GUARD("fvm_compute_update0"); return enq_update0(c); }
int fvm_compute_reconstruction(fvm_ctx *c) { STEP_GUARD("fvm_compute_reconstruction"); return enq_recon(c); }

int fvm_end_step(fvm_ctx *c, int shared) {
  STEP_GUARD("fvm_end_step");
  c->in_step = false;
  int rc = enq_end(c, shared);
  if (rc) return rc;
  if ((rc = read_sched(c))) return rc;
  kt_collect(c);
  c->max_rung = c->hS.iscal[0];
  if ((rc = check_sched_errors(c))) return rc;
  return c->hS.iscal[1];
}

int fvm_step(fvm_ctx *c, int shared) {
  if (!c || !c->have_state) { if (c) c->err = "fvm_step: no state"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_step: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  CK(cudaEventRecord(c->ev0, c->st));
  int rc = enq_step(c, shared);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev1, c->st));
  if ((rc = read_sched(c))) return rc;
  kt_collect(c);
  cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
  c->max_rung = c->hS.iscal[0];
  if ((rc = check_sched_errors(c))) return rc;
  return c->hS.iscal[1];
}

// nsteps steps from one captured CUDA graph per mode, no host round trip
// between steps.  Per-kernel profiling is not recorded in this mode.
int fvm_run(fvm_ctx *c, int nsteps, int shared, long long *faces_out) {
  if (!c || !c->have_state) { if (c) c->err = "fvm_run: no state"; return FVM_ENOMESH; }
  if (c->in_step || nsteps < 0) { c->err = "fvm_run: bad call"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const int g = shared ? 1 : 0;
  if (!c->graph[g]) {
    const bool prof = c->prof;
    c->prof = false;
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    int rc = enq_step(c, shared);
    cudaError_t e = cudaStreamEndCapture(c->st, &gr);
    c->prof = prof;
    if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
    if (e != cudaSuccess) { c->err = std::string("graph capture: ") + cudaGetErrorString(e); return FVM_ECUDA; }
    e = cudaGraphInstantiate(&c->graph[g], gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) { c->graph[g] = nullptr; c->err = std::string("graph instantiate: ") + cudaGetErrorString(e); return FVM_ECUDA; }
  }
  CK(cudaMemcpyAsync(&c->hS, c->d.S, sizeof(Sched), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const unsigned long long a0 = c->hS.nactive_total, f0 = c->hS.nfaces_total;
  CK(cudaEventRecord(c->ev0, c->st));
  for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(c->graph[g], c->st));
  CK(cudaEventRecord(c->ev1, c->st));
  int rc = read_sched(c);
  if (rc) return rc;
  cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
  c->max_rung = c->hS.iscal[0];
  if ((rc = check_sched_errors(c))) return rc;
  if (faces_out) *faces_out = (long long)(c->hS.nfaces_total - f0);
  return (int)(c->hS.nactive_total - a0);
}

double fvm_time(const fvm_ctx *c) { return c ? c->t_global : 0.0; }

void *fvm_stream(fvm_ctx *c) { return c ? (void *)c->st : nullptr; }

int fvm_get_motion(fvm_ctx *c, double *orig_pos, double *orig_vel, float *divb) {
  if (!c || !c->have_mesh) return FVM_ENOMESH;
  CK(cudaSetDevice(c->device));
  const size_t n = c->n;
  if (orig_pos) CK(cudaMemcpyAsync(orig_pos, c->d.opos, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (orig_vel) CK(cudaMemcpyAsync(orig_vel, c->d.ovel, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (divb) CK(cudaMemcpyAsync(divb, c->d.divb, n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int fvm_clock(fvm_ctx *c, unsigned long long *tsys_ticks, double *dt_global, long long *iteration) {
  if (!c || !c->have_state) return FVM_ENOMESH;
  if (c->in_step) { c->err = "fvm_clock: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const int rc = read_sched(c);
  if (rc) return rc;
  if (tsys_ticks) *tsys_ticks = c->hS.tsysU;
  if (dt_global) *dt_global = c->P.dt_tick * (double)(c->hS.tsysU - c->hS.tprevU);
  if (iteration) *iteration = (long long)c->hS.steps;
  return 0;
}

// system::dump_binary (MPI/dump_binary.cpp:5-99) for one rank.  The state is
// brought to the host and converted there with the same to_primitive and
// pressure as the device path, in double precision, then rounded to float as
// the reference's fdump does.
int fvm_dump_binary(fvm_ctx *c, const char *path, const int *idx, const float *rmax) {
  if (!c || !path) return FVM_EINVAL;
  if (!c->have_state) { c->err = "fvm_dump_binary: no state"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_dump_binary: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const size_t n = c->n;
  std::vector<double> U(10 * n), opos(3 * n), ovel(3 * n), vol(n);
  std::vector<float> divb(n);
  std::vector<int> rung(n), bnd(n);
  CK(cudaMemcpyAsync(U.data(), c->d.U, U.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(opos.data(), c->d.opos, opos.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(ovel.data(), c->d.ovel, ovel.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(vol.data(), c->d.cvol, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(divb.data(), c->d.divb, n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(rung.data(), c->d.rung, n * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(bnd.data(), c->d.bnd, n * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  const int rc = read_sched(c);  // synchronises the stream
  if (rc) return rc;

  std::vector<uint32_t> w;
  w.reserve(22 + 28 * n);
  auto iw = [&](int v) { uint32_t u; memcpy(&u, &v, 4); w.push_back(u); };
  auto fw = [&](double v) { const float f = (float)v; uint32_t u; memcpy(&u, &f, 4); w.push_back(u); };
  const Sched &S = c->hS;
  iw(20 * 4);
  iw(0);  // myproc
  iw(1);  // nproc
  iw(1);  // nproc
  w.push_back((uint32_t)(S.tsysU & 0xffffffffULL));
  w.push_back((uint32_t)(S.tsysU >> 32));
  iw(c->n);  // global_n
  iw(c->n);  // local_n
  iw(3);
  fw(S.t_global);
  fw(c->P.dt_tick * (double)(S.tsysU - S.tprevU));  // dt_global
  iw((int)S.steps);                                   // iteration
  fw(c->P.courant);
  fw(c->P.gamma);
  iw(-1);
  for (int a = 0; a < 3; a++) fw(0.0);  // periodic domain [0, box)
  for (int a = 0; a < 3; a++) fw(c->P.box[a]);
  iw(20 * 4);
  for (size_t i = 0; i < n; i++) {
    double W[10];
    to_primitive<double>(&U[10 * i], vol[i], W);
    const double L = std::pow(vol[i] * 3.0 / 4.0 / M_PI, 1.0 / 3.0);
    iw(26 * 4);
    iw(idx ? idx[i] : (int)i);
    for (int a = 0; a < 3; a++) fw(opos[3 * i + a]);
    for (int a = 0; a < 3; a++) fw(ovel[3 * i + a]);
    fw(W[DENS]);
    fw(W[ETHM]);
    fw(pressure<double>(c->P, W));
    fw(rmax ? (double)rmax[i] : 0.0);
    iw(bnd[i]);
    fw(W[VELX]); fw(W[VELY]); fw(W[VELZ]);
    fw(W[BX]); fw(W[BY]); fw(W[BZ]);
    fw(get_dt(c->P, rung[i]));
    fw(vol[i]);
    fw(W[PSI]);
    fw(L * (double)divb[i]);
    fw(W[ENTR]);
    fw(0.0); fw(0.0); fw(0.0);  // J
    iw(26 * 4);
  }
  FILE *f = fopen(path, "wb");
  if (!f) { c->err = std::string("fvm_dump_binary: cannot open ") + path; return FVM_EIO; }
  const size_t put = fwrite(w.data(), sizeof(uint32_t), w.size(), f);
  const int cl = fclose(f);
  if (put != w.size() || cl != 0) { c->err = std::string("fvm_dump_binary: short write to ") + path; return FVM_EIO; }
  return 0;
}

int fvm_last_adjust_stats(const fvm_ctx *c, int *dirty_sites, int *replays, int *sequential) {
  if (!c) return FVM_EINVAL;
  if (dirty_sites) *dirty_sites = c->hS.iscal[4];
  if (replays) *replays = c->hS.iscal[6];
  if (sequential) *sequential = c->hS.iscal[7];
  return 0;
}

// FP64 FMA throughput of the device, the denominator of the FP64 roofline:
// a full-occupancy grid whose threads each run eight independent FMA chains
// (a <- a * m + b, bounded for m < 1).  The final test never holds, so the
// chains are live but nothing is stored.
constexpr int FP64P_CHAINS = 8, FP64P_ITERS = 16384;
__global__ void __launch_bounds__(256) k_fp64_peak(double m, double b, double *sink) {
  double a[FP64P_CHAINS];
#pragma unroll
  for (int k = 0; k < FP64P_CHAINS; k++) a[k] = (double)(threadIdx.x + k) * 1e-3;
#pragma unroll 16
  for (int it = 0; it < FP64P_ITERS; it++)
#pragma unroll
    for (int k = 0; k < FP64P_CHAINS; k++) a[k] = fma(a[k], m, b);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < FP64P_CHAINS; k++) s += a[k];
  if (s == -1.0) *sink = s;
}

int fvm_fp64_peak(fvm_ctx *c, double *flops_per_s) {
  if (!c || !flops_per_s || !c->d.S) { if (c) c->err = "fvm_fp64_peak: bad arguments"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int blocks = sms * 8, threads = 256;
  float best = 0.0f;
  for (int rep = 0; rep < 4; rep++) {  // the first launch warms up; the fastest of the rest counts
    CK(cudaEventRecord(c->ev0, c->st));
    k_fp64_peak<<<blocks, threads, 0, c->st>>>(0.999999, 1e-6, &c->d.S->sink);
    LAUNCH_CHECK();
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (rep > 0 && (best == 0.0f || ms < best)) best = ms;
  }
  const double flops = 2.0 * FP64P_CHAINS * (double)FP64P_ITERS * blocks * threads;
  *flops_per_s = flops / (best * 1e-3);
  return 0;
}

int fvm_last_step_counts(const fvm_ctx *c, int *ncell_active, int *nface_active) {
  if (!c) return FVM_EINVAL;
  if (ncell_active) *ncell_active = c->hS.iscal[1];
  if (nface_active) *nface_active = c->hS.iscal[3];
  return 0;
}
long long fvm_launch_count(const fvm_ctx *c) { return c ? c->launches : 0; }

int fvm_set_profiling(fvm_ctx *c, int on) {
  if (!c) return FVM_EINVAL;
  c->prof = on != 0;
  for (int k = 0; k < KT_COUNT; k++) { c->kt_ms[k] = 0.0; c->kt_calls[k] = 0; c->kev_pending[k] = false; }
  return 0;
}

int fvm_kernel_times(const fvm_ctx *c, int k, const char **name, double *total_ms, long long *calls) {
  if (!c || k < 0) return FVM_EINVAL;
  if (k >= KT_COUNT) return 0;
  if (name) *name = kKernelNames[k];
  if (total_ms) *total_ms = c->kt_ms[k];
  if (calls) *calls = c->kt_calls[k];
  return 1;
}
unsigned long long fvm_tsys_ticks(const fvm_ctx *c) { return c ? c->tsysU : 0ULL; }
float fvm_last_step_ms(const fvm_ctx *c) { return c ? c->last_ms : 0.0f; }

int fvm_get_active_faces(fvm_ctx *c, int *ids, int *nout) {
  if (!c || !c->have_state) return FVM_ENOMESH;
  CK(cudaSetDevice(c->device));
  std::vector<unsigned char> act(c->n);
  std::vector<int> bnd(c->n);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(act.data(), c->d.act, c->n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(bnd.data(), c->d.bnd, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
  std::vector<unsigned char> seen(c->nf > 0 ? c->nf : 1, 0);
  int cnt = 0;
  for (int i = 0; i < c->n; i++) {
    if (!(act[i] & A_ACTIVE) || bnd[i] != NO_BOUNDARY) continue;
    for (long long q = c->h_off[i]; q < c->h_off[i + 1]; q++) {
      const int f = c->h_ids[q];
      if (seen[f]) continue;
      seen[f] = 1;
      if (ids) ids[cnt] = f;
      cnt++;
    }
  }
  if (nout) *nout = cnt;
  return 0;
}

int fvm_get_limited_wrec(fvm_ctx *c, double *wrec) {
  if (!c || !c->have_state || !wrec) return FVM_EINVAL;
  CK(cudaSetDevice(c->device));
  double *tmp = nullptr;
  CK(cudaMalloc(&tmp, 50 * sizeof(double) * (size_t)c->n));
  BULK(k_limited_wrec<R><<<nblk(c->n, 128), 128, 0, c->st>>>(c->n, c->d.act, (const R *)c->d.Wrec,
                                                             (const R *)c->d.tau, tmp));
  cudaError_t e = cudaMemcpyAsync(wrec, tmp, 50 * sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->st);
  cudaStreamSynchronize(c->st);
  cudaFree(tmp);
  if (e != cudaSuccess) { c->err = cudaGetErrorString(e); return FVM_ECUDA; }
  return 0;
}

int fvm_get_step_dU(fvm_ctx *c, double *dU) {
  if (!c || !dU) return FVM_EINVAL;
  if (!c->d.stepdU) { c->err = "fvm_get_step_dU: set FVM_KEEP_STEP_DU before fvm_set_mesh"; return FVM_EINVAL; }
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(dU, c->d.stepdU, 14 * sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost));
  return 0;
}

int fvm_get_dt_list(fvm_ctx *c, double *dt) {
  if (!c || !dt || !c->have_mesh) return FVM_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(dt, c->d.dtl, sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost));
  return 0;
}

int fvm_get_counters(fvm_ctx *c, long long *out2) {
  if (!c || !out2 || !c->have_mesh) return FVM_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  unsigned long long h[2];
  CK(cudaMemcpy(h, c->d.counters, sizeof(h), cudaMemcpyDeviceToHost));
  out2[0] = (long long)h[0];
  out2[1] = (long long)h[1];
  return 0;
}

int fvm_compute_flux(fvm_ctx *c, int nface, const double *wij, const double *Wi, const double *Wj, const int *jbnd,
                     const double *normal, double *psi, double *Bn, double *flux) {
  if (!c || nface < 0 || !wij || !Wi || !Wj || !normal || !psi || !Bn || !flux) return FVM_EINVAL;
  if (nface == 0) return 0;
  CK(cudaSetDevice(c->device));
  const size_t nf = nface;
  const size_t bytes = sizeof(double) * nf * (3 + 10 + 10 + 3 + 1 + 1 + 10) + sizeof(int) * nf;
  char *buf = nullptr;
  CK(cudaMalloc(&buf, bytes));
  double *dw = (double *)buf, *da = dw + 3 * nf, *db = da + 10 * nf, *dn = db + 10 * nf, *dp = dn + 3 * nf,
         *dB = dp + nf, *dF = dB + nf;
  int *dj = (int *)(dF + 10 * nf);
  cudaMemcpyAsync(dw, wij, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(da, Wi, sizeof(double) * 10 * nf, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(db, Wj, sizeof(double) * 10 * nf, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(dn, normal, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, c->st);
  if (jbnd) cudaMemcpyAsync(dj, jbnd, sizeof(int) * nf, cudaMemcpyHostToDevice, c->st);
  k_flux_kat<<<nblk(nface, 128), 128, 0, c->st>>>(nface, c->P, dw, da, db, jbnd ? dj : nullptr, dn, dp, dB, dF);
  cudaMemcpyAsync(psi, dp, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(Bn, dB, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(flux, dF, sizeof(double) * 10 * nf, cudaMemcpyDeviceToHost, c->st);
  cudaError_t e = cudaStreamSynchronize(c->st);
  cudaFree(buf);
  if (e != cudaSuccess) { c->err = cudaGetErrorString(e); return FVM_ECUDA; }
  return 0;
}

}  // extern "C"

// ==================== fvm_compute_flux_static (no allocation) ====================
//
// fvm_compute_flux stages its face batch in a device buffer it cudaMallocs and
// cudaFrees on every call.  Some callers cannot do that while they run: a host
// integrator that solves boundary or sub-grid face batches between steps of a
// GPU pipeline whose other streams stay busy (cudaFree waits for the whole
// device, stalling them), and a run that holds most of HBM for its mesh, where
// a per-call cudaMalloc can fail half way through.  fvm_compute_flux_static
// runs the same kernel (k_flux_kat) on the same inputs with its staging in the
// file-scope array below instead, and calls no allocating routine.
//
// Capacity: FVM_FLUX_STATIC_MAX_FACES faces per call (308 bytes a face, about
// 5 MB, held by every process that loads this library on each device it uses).
// Layout, in doubles unless noted, each region sized for the capacity:
//   wij 3, Wi 10, Wj 10, normal 3, psi 1, Bn 1, flux 10, boundary flags 1 (int)
// The capacity is a multiple of 32, so every region starts 256-byte aligned.
// Only the boundary-flag region must start at zero, and only when the caller
// passes no flags: it is cleared on the stream before the kernel.  Every call
// on a device shares this one array, so calls whose GPU work overlaps (from
// several host threads, or several contexts on one device, at once) race;
// each call returns only after its stream has synchronised, so calls made one
// after another do not overlap.

static_assert(FVM_FLUX_STATIC_MAX_FACES % 32 == 0, "regions of the staging array must stay 256-byte aligned");
#define FLUX_STAGE_DOUBLES_PER_FACE 38
static __device__ __align__(256) double g_flux_stage[(size_t)FVM_FLUX_STATIC_MAX_FACES * FLUX_STAGE_DOUBLES_PER_FACE +
                                                     FVM_FLUX_STATIC_MAX_FACES / 2];

namespace {
constexpr int kStageDevices = 64;
std::mutex g_flux_stage_mu;
double *g_flux_stage_ptr[kStageDevices];  // device address of g_flux_stage, per device

// Device address of the staging array on the current device (looked up once
// per device).  The caller has made c->device current.
int flux_stage_address(fvm_ctx *c, double **out) {
  if (c->device < 0 || c->device >= kStageDevices) {
    c->err = "fvm_compute_flux_static: device index out of range";
    return FVM_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_flux_stage_mu);
  if (!g_flux_stage_ptr[c->device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_flux_stage);
    if (e != cudaSuccess || !p) {
      c->err = std::string("fvm_compute_flux_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return FVM_ECUDA;
    }
    g_flux_stage_ptr[c->device] = (double *)p;
  }
  *out = g_flux_stage_ptr[c->device];
  return 0;
}
}  // namespace

extern "C" {

int fvm_compute_flux_static(fvm_ctx *c, int nface, const double *wij, const double *Wi, const double *Wj,
                            const int *jbnd, const double *normal, double *psi, double *Bn, double *flux) {
  if (!c || nface < 0 || !wij || !Wi || !Wj || !normal || !psi || !Bn || !flux) return FVM_EINVAL;
  if (nface > FVM_FLUX_STATIC_MAX_FACES) {
    c->err = "fvm_compute_flux_static: nface " + std::to_string(nface) + " exceeds the static staging capacity of " +
             std::to_string(FVM_FLUX_STATIC_MAX_FACES) + " faces; split the batch or use fvm_compute_flux";
    return FVM_ERANGE;
  }
  if (nface == 0) return 0;
  CK(cudaSetDevice(c->device));
  double *base = nullptr;
  const int rc = flux_stage_address(c, &base);
  if (rc) return rc;
  const size_t M = FVM_FLUX_STATIC_MAX_FACES, nf = nface;
  double *dw = base, *da = dw + 3 * M, *db = da + 10 * M, *dn = db + 10 * M, *dp = dn + 3 * M, *dB = dp + M,
         *dF = dB + M;
  int *dj = (int *)(dF + 10 * M);
  CK(cudaMemcpyAsync(dw, wij, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(da, Wi, sizeof(double) * 10 * nf, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(db, Wj, sizeof(double) * 10 * nf, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dn, normal, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, c->st));
  if (jbnd)
    CK(cudaMemcpyAsync(dj, jbnd, sizeof(int) * nf, cudaMemcpyHostToDevice, c->st));
  else
    CK(cudaMemsetAsync(dj, 0, sizeof(int) * nf, c->st));
  k_flux_kat<<<nblk(nface, 128), 128, 0, c->st>>>(nface, c->P, dw, da, db, dj, dn, dp, dB, dF);
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaMemcpyAsync(psi, dp, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(Bn, dB, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(flux, dF, sizeof(double) * 10 * nf, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

}  // extern "C"

// ============================ learned flux network ============================

// The network on n rows (or on *n_dev rows, at most nmax, counted on the
// device): persistent CTAs, one per SM, four 128-row tiles in flight in each.
static int mlp_launch_dev(fvm_ctx *c, int nmax, const int *n_dev, const __nv_bfloat16 *X, float *Y) {
  if (nmax <= 0) return 0;
  static bool attr_set[kMaxDevices] = {};  // per device, like the attribute itself
  if (c->device < 0 || c->device >= kMaxDevices) { c->err = "device index out of range"; return FVM_EINVAL; }
  if (!attr_set[c->device]) {
    CK(cudaFuncSetAttribute(mlp::k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::SMEM_BYTES));
    attr_set[c->device] = true;
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int nchains = (nmax + mlp::TILE * mlp::GROUPS - 1) / (mlp::TILE * mlp::GROUPS);
  const int grid = nchains < nsm ? nchains : nsm;
  mlp::k_mlp_infer<<<grid, mlp::THREADS, mlp::SMEM_BYTES, c->st>>>(nmax, n_dev, X, Y, (const uint4 *)c->mlp_img,
                                                          c->mlp_bias, c->mlp_err);
  LAUNCH_CHECK();
  return 0;
}

static int mlp_launch(fvm_ctx *c, int n, const __nv_bfloat16 *X, float *Y) {
  return mlp_launch_dev(c, n, nullptr, X, Y);
}

extern "C" {

int fvm_mlp_set_weights(fvm_ctx *c, const float *params) {
  if (!c || !params) return FVM_EINVAL;
  CK(cudaSetDevice(c->device));
  if (!c->mlp_img) {
    CK(cudaMalloc(&c->mlp_img, mlp::IMG_BYTES));
    CK(cudaMalloc(&c->mlp_bias, mlp::NBIAS * sizeof(float)));
    CK(cudaMalloc(&c->mlp_err, sizeof(int)));
    CK(cudaMalloc(&c->mlp_param, mlp::NPARAM * sizeof(float)));
    CK(cudaMemsetAsync(c->mlp_err, 0, sizeof(int), c->st));
  }
  CK(cudaMemcpyAsync(c->mlp_param, params, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice, c->st));
  mlp::k_mlp_pack<<<(mlp::NH * mlp::NH + 255) / 256, 256, 0, c->st>>>(c->mlp_param, c->mlp_img, c->mlp_bias);
  LAUNCH_CHECK();
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int fvm_mlp_get_weights(fvm_ctx *c, float *params) {
  if (!c || !params) return FVM_EINVAL;
  if (!c->mlp_param) { c->err = "fvm_mlp_get_weights: no weights"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(params, c->mlp_param, mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// ---- training: forward + backward of one batch of `rows` rows ---------------
// Largest K split of a training product (the weight gradients: M, N <= 128,
// K = batch rows), and the partial tiles it needs.
constexpr int kMaxSplit = 64;

struct MlpWork {
  int rows = 0;
  float *X, *T, *Z1, *Z2, *Z3, *Z4, *A1, *A2, *A3, *G, *dA, *dB, *grad, *loss, *wt, *m, *v, *part;
  void *base = nullptr;
};

static int mlp_work(fvm_ctx *c, MlpWork &w, int rows) {
  using namespace mlp;
  const size_t npart = (size_t)kMaxSplit * NH * NH;  // split-K partial tiles of the weight gradients
  const size_t nf = (size_t)rows * (NIN + NOUT + 3 * NH + NOUT + 3 * NH + NOUT + 2 * NH) + 3 * (size_t)NPARAM + 1 + NOUT +
                    npart;
  CK(cudaMallocAsync(&w.base, nf * sizeof(float), c->st));
  CK(cudaMemsetAsync(w.base, 0, nf * sizeof(float), c->st));
  float *p = (float *)w.base;
  auto take = [&](size_t k) { float *q = p; p += k; return q; };
  w.rows = rows;
  w.X = take((size_t)rows * NIN); w.T = take((size_t)rows * NOUT);
  w.Z1 = take((size_t)rows * NH); w.Z2 = take((size_t)rows * NH); w.Z3 = take((size_t)rows * NH);
  w.Z4 = take((size_t)rows * NOUT);
  w.A1 = take((size_t)rows * NH); w.A2 = take((size_t)rows * NH); w.A3 = take((size_t)rows * NH);
  w.G = take((size_t)rows * NOUT); w.dA = take((size_t)rows * NH); w.dB = take((size_t)rows * NH);
  w.grad = take(NPARAM); w.m = take(NPARAM); w.v = take(NPARAM); w.loss = take(1); w.wt = take(NOUT);
  w.part = take(npart);
  // the tensor-core product's shared memory, set once per device
  static bool attr[kMaxDevices] = {};
  if (c->device < 0 || c->device >= kMaxDevices) { c->err = "device index out of range"; return FVM_EINVAL; }
  if (!attr[c->device]) {
    CK(cudaFuncSetAttribute(mlpt::k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, mlpt::TC_SMEM));
    attr[c->device] = true;
  }
  return 0;
}

// C = A B on the tensor cores (mlpt::k_gemm_tc).  Products with one output
// tile and a long K are split over up to kMaxSplit CTAs of at least two
// chunks each and summed in split order.
static void gemm(fvm_ctx *c, const MlpWork &w, int M, int N, int K, const float *A, long long sam, long long sak,
                 const float *B, long long sbk, long long sbn, float *C, int ldc) {
  cudaStream_t s = c->st;
  const int tiles_m = (M + mlpt::TM - 1) / mlpt::TM, tiles_n = (N + mlpt::TN - 1) / mlpt::TN;
  const int nchunk = (K + mlpt::TK - 1) / mlpt::TK;
  int nsplit = 1, cps = nchunk;
  if (tiles_m * tiles_n == 1 && nchunk >= 4) {
    nsplit = std::min(kMaxSplit, nchunk / 2);
    cps = (nchunk + nsplit - 1) / nsplit;
    nsplit = (nchunk + cps - 1) / cps;
  }
  dim3 grid(tiles_n, tiles_m, nsplit);
  mlpt::k_gemm_tc<<<grid, 128, mlpt::TC_SMEM, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, 0, cps, w.part,
                                                   c->mlp_err);
  if (nsplit > 1) mlpt::k_splitk_sum<<<(M * N + 255) / 256, 256, 0, s>>>(M, N, nsplit, w.part, C, ldc, 0);
}

// Loss (added to *w.loss) and gradient (w.grad) of the batch in w.X / w.T at
// the parameters P.
static int mlp_fwd_bwd(fvm_ctx *c, MlpWork &w, const float *P) {
  using namespace mlp;
  const int B = w.rows;
  cudaStream_t s = c->st;
  const float *W1 = P, *b1 = W1 + NH * NIN, *W2 = b1 + NH, *b2 = W2 + NH * NH, *W3 = b2 + NH, *b3 = W3 + NH * NH,
              *W4 = b3 + NH, *b4 = W4 + NOUT * NH;
  float *g = w.grad;
  float *gW1 = g, *gb1 = gW1 + NH * NIN, *gW2 = gb1 + NH, *gb2 = gW2 + NH * NH, *gW3 = gb2 + NH,
        *gb3 = gW3 + NH * NH, *gW4 = gb3 + NH, *gb4 = gW4 + NOUT * NH;
  const long long nh = (long long)B * NH;
  const unsigned eb = (unsigned)((nh + 255) / 256);
  // forward
  gemm(c, w, B, NH, NIN, w.X, NIN, 1, W1, 1, NIN, w.Z1, NH);
  mlpt::k_bias_gelu<<<eb, 256, 0, s>>>(B, NH, w.Z1, b1, w.A1);
  gemm(c, w, B, NH, NH, w.A1, NH, 1, W2, 1, NH, w.Z2, NH);
  mlpt::k_bias_gelu<<<eb, 256, 0, s>>>(B, NH, w.Z2, b2, w.A2);
  gemm(c, w, B, NH, NH, w.A2, NH, 1, W3, 1, NH, w.Z3, NH);
  mlpt::k_bias_gelu<<<eb, 256, 0, s>>>(B, NH, w.Z3, b3, w.A3);
  gemm(c, w, B, NOUT, NH, w.A3, NH, 1, W4, 1, NH, w.Z4, NOUT);
  mlpt::k_out_loss<<<(B * NOUT + 255) / 256, 256, 0, s>>>(B, w.Z4, b4, w.T, w.wt, w.G, w.loss);
  // backward
  gemm(c, w, NOUT, NH, B, w.G, 1, NOUT, w.A3, NH, 1, gW4, NH);
  mlpt::k_colsum<<<1, 32, 0, s>>>(B, NOUT, w.G, gb4);
  gemm(c, w, B, NH, NOUT, w.G, NOUT, 1, W4, NH, 1, w.dA, NH);
  mlpt::k_gelu_back<<<eb, 256, 0, s>>>(nh, w.dA, w.Z3);
  gemm(c, w, NH, NH, B, w.dA, 1, NH, w.A2, NH, 1, gW3, NH);
  mlpt::k_colsum<<<1, NH, 0, s>>>(B, NH, w.dA, gb3);
  gemm(c, w, B, NH, NH, w.dA, NH, 1, W3, NH, 1, w.dB, NH);
  mlpt::k_gelu_back<<<eb, 256, 0, s>>>(nh, w.dB, w.Z2);
  gemm(c, w, NH, NH, B, w.dB, 1, NH, w.A1, NH, 1, gW2, NH);
  mlpt::k_colsum<<<1, NH, 0, s>>>(B, NH, w.dB, gb2);
  gemm(c, w, B, NH, NH, w.dB, NH, 1, W2, NH, 1, w.dA, NH);
  mlpt::k_gelu_back<<<eb, 256, 0, s>>>(nh, w.dA, w.Z1);
  gemm(c, w, NH, NIN, B, w.dA, 1, NH, w.X, NIN, 1, gW1, NIN);
  mlpt::k_colsum<<<1, NH, 0, s>>>(B, NH, w.dA, gb1);
  c->launches += 21;
  CK(cudaGetLastError());
  return 0;
}

static int mlp_set_wt(fvm_ctx *c, MlpWork &w, const float *wt) {
  float h[mlp::NOUT];
  for (int k = 0; k < mlp::NOUT; k++) h[k] = wt ? wt[k] : 1.0f;
  CK(cudaMemcpyAsync(w.wt, h, sizeof(h), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));  // h is on the stack
  return 0;
}

int fvm_mlp_grad(fvm_ctx *c, int n, const float *X, const float *T, const float *wt, float *grad, float *loss) {
  if (!c || n <= 0 || !X || !T || !grad || !loss) return FVM_EINVAL;
  if (!c->mlp_param) { c->err = "fvm_mlp_grad: no weights"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  MlpWork w;
  int rc = mlp_work(c, w, n);
  if (rc) return rc;
  if ((rc = mlp_set_wt(c, w, wt))) return rc;
  CK(cudaMemcpyAsync(w.X, X, (size_t)n * mlp::NIN * sizeof(float), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(w.T, T, (size_t)n * mlp::NOUT * sizeof(float), cudaMemcpyHostToDevice, c->st));
  if ((rc = mlp_fwd_bwd(c, w, c->mlp_param))) return rc;
  CK(cudaMemcpyAsync(grad, w.grad, mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(loss, w.loss, sizeof(float), cudaMemcpyDeviceToHost, c->st));
  int herr = 0;
  CK(cudaMemcpyAsync(&herr, c->mlp_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaFreeAsync(w.base, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (herr & 4) { c->err = "fvm_mlp_grad: tensor-core product wait timed out"; return FVM_ECUDA; }
  return 0;
}

int fvm_mlp_train(fvm_ctx *c, long long n, const float *X, const float *T, const float *wt, int batch, int steps,
                  float lr, unsigned long long seed, float *loss_out) {
  if (!c || n <= 0 || !X || !T || batch <= 0 || steps < 0 || !(lr > 0.0f)) return FVM_EINVAL;
  if (!c->mlp_param) { c->err = "fvm_mlp_train: no initial weights"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  MlpWork w;
  int rc = mlp_work(c, w, batch);
  if (rc) return rc;
  if ((rc = mlp_set_wt(c, w, wt))) return rc;
  float *dX = nullptr, *dT = nullptr, *hist = nullptr;
  CK(cudaMallocAsync(&dX, (size_t)n * mlp::NIN * sizeof(float), c->st));
  CK(cudaMallocAsync(&dT, (size_t)n * mlp::NOUT * sizeof(float), c->st));
  CK(cudaMallocAsync(&hist, (size_t)(steps > 0 ? steps : 1) * sizeof(float), c->st));
  CK(cudaMemcpyAsync(dX, X, (size_t)n * mlp::NIN * sizeof(float), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dT, T, (size_t)n * mlp::NOUT * sizeof(float), cudaMemcpyHostToDevice, c->st));
  const float b1 = 0.9f, b2 = 0.999f;
  double p1 = 1.0, p2 = 1.0;
  for (int it = 0; it < steps; it++) {
    mlpt::k_gather<<<(batch + 127) / 128, 128, 0, c->st>>>(n, dX, dT, batch, seed, it, w.X, w.T);
    CK(cudaMemsetAsync(w.loss, 0, sizeof(float), c->st));
    if ((rc = mlp_fwd_bwd(c, w, c->mlp_param))) return rc;
    p1 *= b1;
    p2 *= b2;
    mlpt::k_adam<<<(mlp::NPARAM + 255) / 256, 256, 0, c->st>>>(mlp::NPARAM, c->mlp_param, w.grad, w.m, w.v, lr, b1,
                                                               b2, 1e-8f, (float)(1.0 - p1), (float)(1.0 - p2));
    CK(cudaMemcpyAsync(hist + it, w.loss, sizeof(float), cudaMemcpyDeviceToDevice, c->st));
    c->launches += 2;
  }
  CK(cudaGetLastError());
  mlp::k_mlp_pack<<<(mlp::NH * mlp::NH + 255) / 256, 256, 0, c->st>>>(c->mlp_param, c->mlp_img, c->mlp_bias);
  LAUNCH_CHECK();
  if (loss_out && steps > 0)
    CK(cudaMemcpyAsync(loss_out, hist, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  int herr = 0;
  CK(cudaMemcpyAsync(&herr, c->mlp_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaFreeAsync(dX, c->st));
  CK(cudaFreeAsync(dT, c->st));
  CK(cudaFreeAsync(hist, c->st));
  CK(cudaFreeAsync(w.base, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (herr & 4) { c->err = "fvm_mlp_train: tensor-core product wait timed out"; return FVM_ECUDA; }
  return 0;
}

int fvm_mlp_eval_counted(fvm_ctx *c, int nmax, int n, const float *X, float *Y) {
  if (!c || nmax < 0 || n < 0 || n > nmax || (nmax > 0 && (!X || !Y))) return FVM_EINVAL;
  if (!c->mlp_img) { c->err = "fvm_mlp_eval_counted: no weights (fvm_mlp_set_weights)"; return FVM_EINVAL; }
  if (nmax == 0) return 0;
  CK(cudaSetDevice(c->device));
  const size_t nx = (size_t)nmax * mlp::NIN, ny = (size_t)nmax * mlp::NOUT;
  float *dx = nullptr, *dy = nullptr;
  __nv_bfloat16 *db = nullptr;
  int *dn = nullptr;
  CK(cudaMallocAsync(&dx, nx * sizeof(float), c->st));
  CK(cudaMallocAsync(&db, nx * sizeof(__nv_bfloat16), c->st));
  CK(cudaMallocAsync(&dy, ny * sizeof(float), c->st));
  CK(cudaMallocAsync(&dn, sizeof(int), c->st));
  CK(cudaMemcpyAsync(dx, X, nx * sizeof(float), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dy, Y, ny * sizeof(float), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dn, &n, sizeof(int), cudaMemcpyHostToDevice, c->st));
  mlp::k_f32_to_bf16<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>((long long)nx, dx, db);
  LAUNCH_CHECK();
  int rc = mlp_launch_dev(c, nmax, dn, db, dy);
  if (rc) return rc;
  CK(cudaMemcpyAsync(Y, dy, ny * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  int herr = 0;
  CK(cudaMemcpyAsync(&herr, c->mlp_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaFreeAsync(dx, c->st));
  CK(cudaFreeAsync(db, c->st));
  CK(cudaFreeAsync(dy, c->st));
  CK(cudaFreeAsync(dn, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (herr) { c->err = "fvm_mlp_eval_counted: tensor-core pipeline wait timed out"; return FVM_ECUDA; }
  return 0;
}

int fvm_mlp_eval(fvm_ctx *c, int n, const float *X, float *Y) {
  if (!c || n < 0 || (n > 0 && (!X || !Y))) return FVM_EINVAL;
  if (!c->mlp_img) { c->err = "fvm_mlp_eval: no weights (fvm_mlp_set_weights)"; return FVM_EINVAL; }
  if (n == 0) return 0;
  CK(cudaSetDevice(c->device));
  const size_t nx = (size_t)n * mlp::NIN, ny = (size_t)n * mlp::NOUT;
  float *dx = nullptr, *dy = nullptr;
  __nv_bfloat16 *db = nullptr;
  CK(cudaMallocAsync(&dx, nx * sizeof(float), c->st));
  CK(cudaMallocAsync(&db, nx * sizeof(__nv_bfloat16), c->st));
  CK(cudaMallocAsync(&dy, ny * sizeof(float), c->st));
  CK(cudaMemcpyAsync(dx, X, nx * sizeof(float), cudaMemcpyHostToDevice, c->st));
  mlp::k_f32_to_bf16<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>((long long)nx, dx, db);
  LAUNCH_CHECK();
  int rc = mlp_launch(c, n, db, dy);
  if (rc) return rc;
  CK(cudaMemcpyAsync(Y, dy, ny * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  int herr = 0;
  CK(cudaMemcpyAsync(&herr, c->mlp_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaFreeAsync(dx, c->st));
  CK(cudaFreeAsync(db, c->st));
  CK(cudaFreeAsync(dy, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (herr) { c->err = "fvm_mlp_eval: tensor-core pipeline wait timed out"; return FVM_ECUDA; }
  return 0;
}

}  // extern "C"

extern "C" {

int fvm_set_flux_mode(fvm_ctx *c, int mode, float drho, float dp, float mach, int judge, int hstride,
                      long long hcap) {
  if (!c || mode < 0 || mode > 2 || judge < 0 || hstride < 1 || hcap < 0) return FVM_EINVAL;
  if (!c->have_mesh) { c->err = "fvm_set_flux_mode: no mesh"; return FVM_ENOMESH; }
  if (mode == 1 && !c->mlp_img) { c->err = "fvm_set_flux_mode: no network weights"; return FVM_EINVAL; }
  if (!(drho >= 0.0f) || !(dp >= 0.0f) || !(mach >= 0.0f)) { c->err = "fvm_set_flux_mode: bad gate"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);
  Dev &d = c->d;
  const size_t nf = (size_t)(c->nf > 0 ? c->nf : 1);
  int rc = 0;
  if (!d.lX) {
    rc |= dalloc_bytes(c, &d.lX, nf * 16 * sizeof(__nv_bfloat16));
    rc |= dalloc_bytes(c, &d.lY, nf * 8 * sizeof(float));
    rc |= dalloc_bytes(c, &d.lface, nf * sizeof(int));
    rc |= dalloc_bytes(c, &d.lcount, sizeof(int));
    rc |= dalloc_bytes(c, &d.lstats, LSTAT_COUNT * sizeof(double));
    rc |= dalloc_bytes(c, &d.lhcount, sizeof(unsigned long long));
    rc |= dalloc_bytes(c, &d.lnorm, 48 * sizeof(float));
  }
  if (mode == 2 && hcap > c->lb.hcap) {
    rc |= dalloc_bytes(c, &d.lhx, (size_t)hcap * 16 * sizeof(float));
    rc |= dalloc_bytes(c, &d.lhy, (size_t)hcap * 8 * sizeof(float));
  }
  if (rc) return FVM_ENOMEM;
  LearnBuf &lb = c->lb;
  lb.X = (__nv_bfloat16 *)d.lX;
  lb.Y = (float *)d.lY;
  lb.gface = (int *)d.lface;
  lb.count = (int *)d.lcount;
  lb.stats = (double *)d.lstats;
  lb.hcount = (unsigned long long *)d.lhcount;
  if (mode == 2 && hcap > lb.hcap) {
    lb.hx = (float *)d.lhx;
    lb.hy = (float *)d.lhy;
    lb.hcap = hcap;
  }
  lb.hstride = (unsigned)hstride;
  lb.judge = (unsigned)judge;
  lb.U = d.U;
  lb.vol = d.cvol;
  lb.norm = (const float *)d.lnorm;
  CK(cudaMemcpy(d.lnorm, c->h_norm, sizeof(c->h_norm), cudaMemcpyHostToDevice));
  lb.drho = drho;
  lb.dp = dp;
  lb.mach = mach;
  CK(cudaMemsetAsync(lb.stats, 0, LSTAT_COUNT * sizeof(double), c->st));
  CK(cudaMemsetAsync(lb.hcount, 0, sizeof(unsigned long long), c->st));
  CK(cudaMemsetAsync(lb.count, 0, sizeof(int), c->st));
  CK(cudaStreamSynchronize(c->st));
  c->learn_mode = mode;
  return 0;
}

int fvm_set_flux_surrogate(fvm_ctx *c, int kind) {
  if (!c || kind < SUR_NETWORK || kind > SUR_LLF) return FVM_EINVAL;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);  // captured steps hold the flux settings by value
  c->lb.surrogate = kind;
  return 0;
}

int fvm_mlp_set_norm(fvm_ctx *c, const float *mu_x, const float *sd_x, const float *mu_y, const float *sd_y) {
  if (!c || !mu_x || !sd_x || !mu_y || !sd_y) return FVM_EINVAL;
  for (int k = 0; k < 16; k++)
    if (!(sd_x[k] > 0.0f)) { c->err = "fvm_mlp_set_norm: feature spreads must be positive"; return FVM_EINVAL; }
  for (int k = 0; k < 16; k++) { c->h_norm[k] = mu_x[k]; c->h_norm[16 + k] = 1.0f / sd_x[k]; }
  for (int k = 0; k < 8; k++) { c->h_norm[32 + k] = mu_y[k]; c->h_norm[40 + k] = sd_y[k]; }
  if (c->d.lnorm) {
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaMemcpy(c->d.lnorm, c->h_norm, sizeof(c->h_norm), cudaMemcpyHostToDevice));
  }
  return 0;
}

int fvm_learn_stats(fvm_ctx *c, double *stats) {
  if (!c || !stats) return FVM_EINVAL;
  if (!c->lb.stats) { for (int k = 0; k < LSTAT_COUNT; k++) stats[k] = 0.0; return 0; }
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(stats, c->lb.stats, LSTAT_COUNT * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

long long fvm_harvest_count(fvm_ctx *c) {
  if (!c || !c->lb.hcount) return 0;
  unsigned long long h = 0;
  if (cudaMemcpyAsync(&h, c->lb.hcount, sizeof(h), cudaMemcpyDeviceToHost, c->st) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(c->st) != cudaSuccess) return -1;
  return (long long)(h < (unsigned long long)c->lb.hcap ? h : (unsigned long long)c->lb.hcap);
}

int fvm_get_harvest(fvm_ctx *c, long long n, float *X, float *Y) {
  if (!c || n < 0 || (n > 0 && (!X || !Y))) return FVM_EINVAL;
  if (n > c->lb.hcap) { c->err = "fvm_get_harvest: more rows than harvested"; return FVM_ERANGE; }
  if (n == 0) return 0;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(X, c->lb.hx, (size_t)n * 16 * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(Y, c->lb.hy, (size_t)n * 8 * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

}  // extern "C"

// ================================ autotuner ================================

namespace {
// The mutable per-cell state of a context (everything a step writes that
// outlives the step), for trial steps that leave no trace.
struct StateCopy {
  std::vector<std::pair<void *, size_t>> items;
  void *buf = nullptr;
};

int state_items(fvm_ctx *c, StateCopy &sc) {
  Dev &d = c->d;
  const size_t n = c->n, rb = c->rb;
  sc.items = {{d.U, 10 * n * 8}, {d.dU, 14 * n * 8}, {d.Wrec, 50 * n * rb}, {d.vel, 3 * n * 8},
              {d.tlast, n * 8},  {d.tend, n * 8},    {d.rung, n * 4},        {d.opos, 3 * n * 8},
              {d.ovel, 3 * n * 8}, {d.divb, n * 4},  {d.volp, n * 8},        {d.mnmx, 20 * n * rb},
              {d.mz, n},           {d.S, sizeof(Sched)}, {d.counters, 4 * sizeof(unsigned long long)}};
  if (d.lstats) sc.items.push_back({d.lstats, LSTAT_COUNT * sizeof(double)});
  size_t total = 0;
  for (auto &it : sc.items) total += (it.second + 255) & ~(size_t)255;
  CK(cudaMallocAsync(&sc.buf, total, c->st));
  return 0;
}

int state_copy(fvm_ctx *c, StateCopy &sc, bool save) {
  char *p = (char *)sc.buf;
  for (auto &it : sc.items) {
    if (save) CK(cudaMemcpyAsync(p, it.first, it.second, cudaMemcpyDeviceToDevice, c->st));
    else CK(cudaMemcpyAsync(it.first, p, it.second, cudaMemcpyDeviceToDevice, c->st));
    p += (it.second + 255) & ~(size_t)255;
  }
  return 0;
}
}  // namespace

extern "C" {

int fvm_set_tuning(fvm_ctx *c, const int *choice) {
  if (!c || !choice) return FVM_EINVAL;
  auto block_ok = [](int b) { return b == 32 || b == 64 || b == 128; };
  if ((choice[0] != 0 && choice[0] != 1) || !block_ok(choice[1]) || !block_ok(choice[2]) || !block_ok(choice[3])) {
    c->err = "fvm_set_tuning: staged limiter must be 0 or 1 and block sizes 32, 64 or 128";
    return FVM_EINVAL;
  }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);  // captured steps hold the launch shapes
  c->tune.lim_staged = choice[0];
  c->tune.bs_face = choice[1];
  c->tune.bs_cell = choice[2];
  c->tune.bs_cell2 = choice[3];
  return 0;
}

int fvm_autotune(fvm_ctx *c, int shared, int steps, int *choice) {
  if (!c || steps < 1) return FVM_EINVAL;
  if (!c->have_state || c->in_step) { c->err = "fvm_autotune: no state, or inside a step"; return FVM_ENOMESH; }
  CK(cudaSetDevice(c->device));
  StateCopy sc;
  int rc = state_items(c, sc);
  if (rc) return rc;
  if ((rc = state_copy(c, sc, true))) return rc;
  const bool prof = c->prof;
  const unsigned long long tsys0 = c->tsysU;
  const double t0 = c->t_global;
  // one trial: `steps` eager steps with per-kernel events, then the state back
  auto trial = [&](double *ms_out) -> int {
    int r = fvm_set_profiling(c, 1);
    if (r) return r;
    for (int s = 0; s < steps; s++) {
      r = fvm_step(c, shared);
      if (r < 0) return r;
    }
    for (int k = 0; k < KT_COUNT; k++) ms_out[k] = c->kt_ms[k];
    if ((r = state_copy(c, sc, false))) return r;
    CK(cudaStreamSynchronize(c->st));
    c->tsysU = tsys0;
    c->t_global = t0;
    return read_sched(c);
  };
  double ms[KT_COUNT];
  // coordinate search, one family at a time, timed on its own kernels
  struct Knob { int *v; int ncand; int cand[3]; int k1, k2; } knobs[] = {
      {&c->tune.lim_staged, 2, {1, 0, 0}, KT_LIMITER, KT_LIMITER},
      {&c->tune.bs_face, 3, {128, 64, 32}, KT_CORR_FLUX, KT_PRED_FLUX},
      {&c->tune.bs_cell, 3, {128, 64, 32}, KT_CORR_CELL, KT_PRED_CELL},
      {&c->tune.bs_cell2, 3, {128, 64, 32}, KT_RECON, KT_LIMITER},
  };
  for (auto &kb : knobs) {
    double best = 1e300;
    int bestv = *kb.v;
    for (int ci = 0; ci < kb.ncand; ci++) {
      const int v = kb.cand[ci];
      *kb.v = v;
      drop_graphs(c);
      if ((rc = trial(ms)) != 0) { c->prof = prof; return rc; }
      const double t = ms[kb.k1] + (kb.k2 != kb.k1 ? ms[kb.k2] : 0.0);
      if (t < best) { best = t; bestv = v; }
    }
    *kb.v = bestv;
  }
  drop_graphs(c);
  fvm_set_profiling(c, prof ? 1 : 0);
  CK(cudaFreeAsync(sc.buf, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (choice) {
    choice[0] = c->tune.lim_staged;
    choice[1] = c->tune.bs_face;
    choice[2] = c->tune.bs_cell;
    choice[3] = c->tune.bs_cell2;
  }
  return 0;
}

}  // extern "C"
