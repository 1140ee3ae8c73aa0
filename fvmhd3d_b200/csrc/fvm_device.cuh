// Device code of the fluid hot path: the step's data layout (Sched, Dev),
// the per-cell and per-face work of every stage as device functions, and the
// stage kernels that launch them.  Included by fvm_kernels.cu (the stage
// kernels and the C-ABI context) and by fvm_fused.cu (the persistent rung
// kernel).  FVM_RESTRICT is __restrict__ unless the including file defines
// it: the persistent kernel reads data that earlier phases of the same
// launch wrote, so its copy of these functions makes no read-only promise.
#pragma once
#include "fvm_math.cuh"
#include "flux_mlp.cuh"
#include "flux_learn.cuh"

#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>

#ifndef FVM_RESTRICT
#define FVM_RESTRICT __restrict__
#endif

namespace fvm {
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
  unsigned long long fused_steps;  // steps run by the persistent rung kernel
  int inc[2];  // incremental list building: [0] links of the active cells, [1] 1 when
               // this step's lists were built that way
  unsigned long long inc_steps;  // steps whose lists were built incrementally
};

struct Dev {
  // mesh
  int2 *s12;
  double4 *geo, *cen, *dr1, *dr2;
  double *cvol, *ccen;
  double *hcell;  // (cvol / (4 pi / 3))^(1/3), Params::hcell
  unsigned char *halo;  // copies of other ranks' cells (Params::halo when set)
  int *off, *lnk;
  int *perm;  // thread slot -> cell (face-count order inside windows of CPW cells)
  int *alist, *bcount;  // ordered active-site list and block offsets (individual timesteps)
  int *flist, *fbcount; // ordered active-face list and its block offsets (partial steps)
  int *clist, *cbcount; // ordered list of the step's active and neighbour cells, block offsets (partial steps)
  int *ilist;           // the step's active cells, unordered (incremental list building)
  unsigned *ibits;      // one bit per cell, zero between steps (incremental list building)
  int *icount;          // per block of k_inc_count / k_site_count: its count (SITE_BLOCKS)
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

}  // namespace fvm

using namespace fvm;

// Minimum resident 128-thread blocks per SM for the face-flux kernels (caps
// their registers): 3 (168 registers, FP64) or 4 (128, FP32).
//
// FP32 global steps (every cell active) launch their own instantiations of
// the exact face passes, the compute_update / compute_update0 cell passes,
// the limiter and the reconstruction, with more resident blocks: the extra
// warps hide more of the gathers than the spills cost (128^3 blast: exact
// flux at 6 blocks, 80 registers: corrector 0.85 -> 0.69 ms, predictor
// 0.80 -> 0.63 ms).  Partial steps keep the instantiations whose bits the
// persistent rung kernel reproduces: the compiler may contract a multiply
// and an add differently when the register budget changes, so a kernel
// compiled to another budget need not give the same last bit.  FP64 keeps
// one set of instantiations: at 4 blocks its face passes were 7-9% faster,
// but the 32^3 Alfven wave's reconstruction then drifted from the oracle
// by 1.18e-12 in ten steps, past the 1e-12 parity bound.
#ifndef FVM_FLUX_MINB_D
#define FVM_FLUX_MINB_D 3
#endif
#ifndef FVM_FLUX_MINB_F
#define FVM_FLUX_MINB_F 4
#endif
#ifndef FVM_GLOBAL_FLUX_MINB_D
#define FVM_GLOBAL_FLUX_MINB_D FVM_FLUX_MINB_D
#endif
#ifndef FVM_GLOBAL_FLUX_MINB_F
#define FVM_GLOBAL_FLUX_MINB_F 6
#endif
#define FVM_FLUX_MINB(R) (sizeof(R) == 4 ? FVM_FLUX_MINB_F : FVM_FLUX_MINB_D)
#define FVM_GLOBAL_FLUX_MINB(R) (sizeof(R) == 4 ? FVM_GLOBAL_FLUX_MINB_F : FVM_GLOBAL_FLUX_MINB_D)
#ifndef FVM_CELL_LFJ
#define FVM_CELL_LFJ 1  // cell kernels take (face, neighbour) from the link table instead of s12
#endif
// Resident blocks per SM that the FP32 global-step instantiations of the
// compute_update and compute_update0 cell passes ask for.  Measured on the
// 128^3 blast: corrector cells 1.04 -> 0.78 ms and predictor cells 0.77 ->
// 0.74 ms at 5 (96 registers, a few bytes of spills).  FP64 global steps
// launch the partial-step kernels (the FP64 instantiations of the global
// ones are built but not launched).
#ifndef FVM_CORR_CELL_MINB_F
#define FVM_CORR_CELL_MINB_F 5
#endif
#ifndef FVM_PRED_CELL_MINB_F
#define FVM_PRED_CELL_MINB_F 5
#endif
#define FVM_CORR_CELL_MINB(R) (sizeof(R) == 4 ? FVM_CORR_CELL_MINB_F : 1)
#define FVM_PRED_CELL_MINB(R) (sizeof(R) == 4 ? FVM_PRED_CELL_MINB_F : 1)
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

__device__ __forceinline__ bool face_active(const unsigned char *act, const int *bnd, int a, int b) {
  return ((act[a] & A_ACTIVE) && bnd[a] == NO_BOUNDARY) || ((act[b] & A_ACTIVE) && bnd[b] == NO_BOUNDARY);
}

__device__ __forceinline__ void ld3(const double *p, double *o) { o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; }

// ---- begin_step: active flags (Scheduler::pull_active_list) ---------------
// Active flags of the step's cells (MPI/Scheduler.h:108-154 picks the rungs)
// and their count.  With ilist, the active cells are also listed (in block
// order) and the links of all of them counted in *ilinks, for the
// incremental list building of a partial step.
__global__ void k_active(int n, const int *FVM_RESTRICT rung, const Sched *FVM_RESTRICT S,
                         unsigned char *FVM_RESTRICT act, int *FVM_RESTRICT nactive, const int *FVM_RESTRICT off,
                         int *FVM_RESTRICT ilist, int *FVM_RESTRICT ilinks) {
  const unsigned long long flags = S->flags;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  bool a = false;
  int links = 0;
  if (i < n) {
    const int r = rung[i];
    a = r >= 0 && r < RUNGMAX && ((flags >> (RUNGMAX - 1 - r)) & 1ULL);
    act[i] = a ? A_ACTIVE : 0;
    if (a && ilist) links = off[i + 1] - off[i];
  }
  __shared__ int wcnt[32], wlinks[32], base;
  const unsigned ballot = __ballot_sync(0xffffffffu, a);
  for (int o = 16; o > 0; o >>= 1) links += __shfl_xor_sync(0xffffffffu, links, o);
  if (lane == 0) { wcnt[wid] = __popc(ballot); wlinks[wid] = links; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0, tl = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      const int cw = wcnt[w];
      wcnt[w] = tot;  // exclusive prefix: the warp's first slot in the block
      tot += cw;
      tl += wlinks[w];
    }
    base = tot ? atomicAdd(nactive, tot) : 0;
    if (ilist && tl) atomicAdd(ilinks, tl);
  }
  __syncthreads();
  if (a && ilist) {
    const int slot = base + wcnt[wid] + __popc(ballot & ((1u << lane) - 1u));
    ilist[slot] = i;
  }
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
__global__ void k_faceflags(int nf, const int2 *FVM_RESTRICT s12, unsigned char *FVM_RESTRICT act,
                            const int *FVM_RESTRICT bnd, unsigned char *FVM_RESTRICT fflag,
                            int *FVM_RESTRICT nface_active, unsigned char *FVM_RESTRICT fcode,
                            unsigned char *FVM_RESTRICT fcode2, int *FVM_RESTRICT bcount) {
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

// ---- incremental list building ---------------------------------------------
// A partial step with few active cells builds the flags and lists of
// k_faceflags and the compactions from the active cells' links, without a
// pass over every face and cell.  The involved cells are the active cells and
// their neighbours; the faces whose flags and codes the step reads are the
// links of those cells, and k_inc_faces rewrites exactly those (a face outside
// them keeps what an earlier step left; k_faceflags treats it as it treats
// every face, and an incremental step that reaches it rewrites it first).
// The involved-cell list comes out in ascending order, as k_place_cells
// leaves it (the adjust_timesteps sites are taken from it in that order);
// the active-face list holds the same faces as k_place_faces leaves, in the
// order they were found: every face pass computes each face on its own.

// The neighbour marks of k_faceflags (an inactive neighbour of an active cell
// is a local neighbour, the active cell has one), and the involved cells as
// bits of ibits.  One warp per active cell, a lane per link.
__global__ void k_inc_mark(const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, unsigned char *act,
                           const Sched *FVM_RESTRICT S, const int *FVM_RESTRICT ilist, unsigned *FVM_RESTRICT ibits) {
  const int na = S->iscal[1], lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int u = w0; u < na; u += nw) {
    const int c = ilist[u], q1 = off[c + 1];
    bool ngb = false;
    for (int q = off[c] + lane; q < q1; q += 32) {
      const int jy = lfj[q].y, j = jy >= 0 ? jy : ~jy;
      if (!(act[j] & A_ACTIVE)) {  // the active bit never changes in this kernel
        act[j] = A_LNGB;
        ngb = true;
        atomicOr(&ibits[j >> 5], 1u << (j & 31));
      }
    }
    if (__any_sync(0xffffffffu, ngb) && lane == 0) act[c] = A_ACTIVE | A_HASNGB;
    if (lane == 0) atomicOr(&ibits[c >> 5], 1u << (c & 31));
  }
}

// The involved cells in ascending order from ibits (clist, count ninv),
// clearing the bits read, in two launches of INC_BLOCKS blocks: block b
// takes the words [b W, (b + 1) W), W a multiple of its thread count, and
// each thread a run of consecutive words.  k_inc_count counts each block's
// bits; k_inc_cells places them after the counts of the blocks before it.
constexpr int INC_BLOCKS = 64;
__device__ __forceinline__ void inc_words(int n, int &w0, int &w1) {
  const int nw = (n + 31) >> 5;
  const int W = ((nw + INC_BLOCKS - 1) / INC_BLOCKS + blockDim.x - 1) / blockDim.x * blockDim.x;
  const int per = W / blockDim.x;
  w0 = blockIdx.x * W + threadIdx.x * per;
  w1 = min(nw, w0 + per);
}
__device__ __forceinline__ int block_sum(int v, int *wsum) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) wsum[wid] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += wsum[w];
  return t;
}
__global__ void __launch_bounds__(256) k_inc_count(int n, const unsigned *FVM_RESTRICT ibits,
                                                   int *FVM_RESTRICT bcnt) {
  __shared__ int wsum[8];
  int w0, w1;
  inc_words(n, w0, w1);
  int c = 0;
  for (int w = w0; w < w1; w++) c += __popc(ibits[w]);
  const int t = block_sum(c, wsum);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = t;
}
__global__ void __launch_bounds__(256) k_inc_cells(int n, Sched *FVM_RESTRICT S, unsigned *FVM_RESTRICT ibits,
                                                   const int *FVM_RESTRICT bcnt, int *FVM_RESTRICT clist) {
  __shared__ int wsum[8], base;
  if (threadIdx.x < 32) {  // the counts of the blocks before this one, and of all
    int before = 0, all = 0;
    for (int b = threadIdx.x; b < INC_BLOCKS; b += 32) {
      const int v = bcnt[b];
      all += v;
      before += b < (int)blockIdx.x ? v : 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
      before += __shfl_xor_sync(0xffffffffu, before, o);
      all += __shfl_xor_sync(0xffffffffu, all, o);
    }
    if (threadIdx.x == 0) {
      base = before;
      if (blockIdx.x == 0) S->ninv = all;
    }
  }
  int w0, w1;
  inc_words(n, w0, w1);
  int c = 0;
  for (int w = w0; w < w1; w++) c += __popc(ibits[w]);
  // exclusive scan of c over the block's threads
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = c;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  int pos = base + x - c;
  for (int w = 0; w < wid; w++) pos += wsum[w];
  for (int w = w0; w < w1; w++) {
    unsigned v = ibits[w];
    if (!v) continue;
    ibits[w] = 0u;
    while (v) {
      clist[pos++] = 32 * w + __ffs(v) - 1;
      v &= v - 1u;
    }
  }
}

// Flags and codes of every face of the involved cells as k_faceflags sets
// them (an inactive face is coded F_OFF), and the active faces, each listed
// once: by its s1 cell when that cell is active and not a boundary cell, else
// by its s2 cell.  One warp per involved cell, a lane per link.
__global__ void k_inc_faces(const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
                            const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
                            unsigned char *FVM_RESTRICT fflag, unsigned char *FVM_RESTRICT fcode,
                            unsigned char *FVM_RESTRICT fcode2, Sched *FVM_RESTRICT S, const int *FVM_RESTRICT clist,
                            int *FVM_RESTRICT flist) {
  const int nc = S->ninv, lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int u = w0; u < nc; u += nw) {
    const int c = clist[u], q1 = off[c + 1];
    const bool cact = act[c] & A_ACTIVE;
    for (int q = off[c] + lane; q < q1; q += 32) {
      const int f = lfj[q].x;
      const int2 e = s12[f];
      const bool a1 = act[e.x] & A_ACTIVE, a2 = act[e.y] & A_ACTIVE;
      const bool b1 = bnd[e.x] != NO_BOUNDARY, b2 = bnd[e.y] != NO_BOUNDARY;
      const bool own1 = a1 && !b1, a = own1 || (a2 && !b2);
      fflag[f] = (unsigned char)((a ? FF_ACTIVE : 0) | (b1 ? FF_BND1 : 0) | (b2 ? FF_BND2 : 0));
      if (!a) {
        fcode[f] = F_OFF;
        fcode2[f] = F_OFF;
      } else if (cact && c == (own1 ? e.x : e.y)) {
        flist[atomicAdd(&S->iscal[3], 1)] = f;
      }
    }
  }
}

// Face offsets used by every face loop, computed once per generator layout:
//   dr1 = centroid - x_s1 (the reference's dri, MPI/compute_update.cpp:136)
//         with w = dri . n (dsh, :164)
//   dr2 = wrap(centroid - x_s2) (MPI/compute_reconstruction.cpp:74-83 seen
//         from s2)
__global__ void k_face_geom(int nf, Params P, const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo,
                            const double4 *FVM_RESTRICT cen, const double *FVM_RESTRICT pos,
                            double4 *FVM_RESTRICT dr1, double4 *FVM_RESTRICT dr2) {
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
__global__ void k_link_recon(int n, Params P, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                             const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
                             const double4 *FVM_RESTRICT dr2, R *FVM_RESTRICT lrw, R *FVM_RESTRICT lrd,
                             R *FVM_RESTRICT lld) {
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
#ifndef FVM_LIMITER_MINB_D
#define FVM_LIMITER_MINB_D 6
#endif
  static constexpr int KH_LIM = 2, MINB_LIM = FVM_LIMITER_MINB_D, KH_REC = 2, MINB_REC = FVM_RECON_MINB_D;
  static constexpr int MINB_LIM_G = MINB_LIM, MINB_REC_G = MINB_REC;  // global steps: the same
};
template <> struct CellTune<float> {
// global steps: 8 blocks for the reconstruction (64 registers, a few
// spills) and 10 for the limiter (46) beat 6 and 8 (128^3 blast: 1.085 ->
// 1.027 ms and 0.915 -> 0.886 ms)
#ifndef FVM_RECON_MINB_F
#define FVM_RECON_MINB_F 8
#endif
#ifndef FVM_LIMITER_MINB_F
#define FVM_LIMITER_MINB_F 10
#endif
  static constexpr int KH_LIM = 2, MINB_LIM = 8, KH_REC = 5, MINB_REC = 6;
  static constexpr int MINB_LIM_G = FVM_LIMITER_MINB_F, MINB_REC_G = FVM_RECON_MINB_F;
};

// KH consecutive bulk values from p, as 2-wide loads when KH is even: the
// callers' rows (10 or 50 values per cell, 6 per link) and even offsets then
// start on 16-byte (FP64) or 8-byte (FP32) boundaries.
template <typename R> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float2; };
template <typename R, int N>
__device__ __forceinline__ void load_n(const R *FVM_RESTRICT p, R *v) {
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
__device__ __forceinline__ void store_n(R *FVM_RESTRICT p, const R *v) {
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
__device__ __forceinline__ void store_contrib(R *FVM_RESTRICT o, const R *v) {
  using V = typename Vec2<R>::T;
  V *o2 = reinterpret_cast<V *>(o);
#pragma unroll
  for (int h = 0; h < 7; h++) { V x; x.x = v[2 * h]; x.y = v[2 * h + 1]; o2[h] = x; }
}

template <typename R, int KH>
__device__ __forceinline__ void limiter_thread(int i, int k0, bool reuse, double t_global,
    const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1, const unsigned char *FVM_RESTRICT fflag,
    const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT tlast,
    const R *FVM_RESTRICT Wrec, R *FVM_RESTRICT tau, R *FVM_RESTRICT fst,
    const R *FVM_RESTRICT mnmx, const unsigned char *FVM_RESTRICT mz, const R *FVM_RESTRICT lld) {
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

// limiter_thread with G lanes (a group of consecutive lanes, gl this lane's
// index, gmask the group's lanes) for one cell and primitive pair, in a step
// where not every cell is active (pass 1 always runs): the faces are split
// among the lanes in passes 1 and 3; the neighbour minimum and maximum of
// pass 1 do not depend on the order (only their magnitudes are used) and are
// reduced by shuffles; pass 2's ratio minimum compares cross-multiplied
// products, whose rounding makes it depend on the order, so every lane folds
// the faces in face order, each face's extrapolated difference taken by
// shuffle from the lane that computed it.  The same bits as limiter_thread.
template <typename R, int KH, int G>
__device__ __forceinline__ void limiter_group(int i, int k0, int gl, unsigned gmask, double t_global,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const unsigned char *FVM_RESTRICT fflag,
    const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT tlast,
    const R *FVM_RESTRICT Wrec, R *FVM_RESTRICT tau, R *FVM_RESTRICT fst, const R *FVM_RESTRICT lld) {
  if (!(act[i] & (A_ACTIVE | A_LNGB))) return;
  const double ti = tlast[i];
  const R *ri = Wrec + 50 * (size_t)i + k0;
  R mn[KH], mx[KH], ln[KH], lq[KH], wi[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { mn[k] = R(0); mx[k] = R(0); ln[k] = R(2); lq[k] = R(1); wi[k] = ri[k]; }
  const int q0 = off[i], q1 = off[i + 1];
  bool zero = false;
  for (int q = q0 + gl; q < q1; q += G) {
    const int2 fj = lfj[q];
    const int f = fj.x, j = fj.y >= 0 ? fj.y : ~fj.y;
    const unsigned char ff = fflag[f];
    if (!(ff & FF_ACTIVE)) continue;
    if (ff & (FF_BND1 | FF_BND2)) { zero = true; continue; }
    R rj[KH];
    load_n<R, KH>(Wrec + 50 * (size_t)j + k0, rj);
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R diff = rj[k] - wi[k];
      mn[k] = smin(mn[k], diff);
      mx[k] = smax(mx[k], diff);
    }
  }
  for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < KH; k++) {
      mn[k] = smin(mn[k], __shfl_xor_sync(gmask, mn[k], o, G));
      mx[k] = smax(mx[k], __shfl_xor_sync(gmask, mx[k], o, G));
    }
  }
  zero = __any_sync(gmask, zero);
  R *to = tau + 10 * (size_t)i + k0;
  R gx[KH], gy[KH], gz[KH], gt[KH];
  if (zero) {
#pragma unroll
    for (int k = 0; k < KH; k++) { if (gl == 0) to[k] = R(0); gx[k] = gy[k] = gz[k] = gt[k] = R(0); }
  } else {
    R thr[KH];
#pragma unroll
    for (int k = 0; k < KH; k++) {
      gx[k] = ri[10 + k]; gy[k] = ri[20 + k]; gz[k] = ri[30 + k]; gt[k] = ri[40 + k];
      thr[k] = limiter_thr(mn[k], mx[k]);
    }
    for (int base = q0; base < q1; base += G) {
      const int q = base + gl;
      R dW[KH];
      int fa = 0;
#pragma unroll
      for (int k = 0; k < KH; k++) dW[k] = R(0);
      if (q < q1) {
        const int2 fj = lfj[q];
        const int f = fj.x;
        if (fflag[f] & FF_ACTIVE) {
          fa = 1;
          const bool own = fj.y >= 0;
          const double tj = tlast[own ? fj.y : ~fj.y];
          const double dtI = t_global - (own ? ti : tj), dtJ = t_global - (own ? tj : ti);
          const double dth = 0.5 * smin(dtI, dtJ);
          const R *l3 = lld + 3 * (size_t)q;
          const R dr[3] = {l3[0], l3[1], l3[2]};
          const R dtt = R(own ? dtI - dth : dtJ - dth);
#pragma unroll
          for (int k = 0; k < KH; k++) {
            const R dWx = gx[k] * dr[0] + gy[k] * dr[1] + gz[k] * dr[2];
            dW[k] = dWx + gt[k] * dtt;
          }
        }
      }
      const int m = min(G, q1 - base);
      for (int jj = 0; jj < m; jj++) {
        const int faj = __shfl_sync(gmask, fa, jj, G);
#pragma unroll
        for (int k = 0; k < KH; k++) {
          const R d = __shfl_sync(gmask, dW[k], jj, G);
          if (faj) limiter_ratio(ln[k], lq[k], d, mn[k], mx[k], thr[k]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const R tk = limiter_finish(ln[k], lq[k]);
      if (gl == 0) to[k] = tk;
      gx[k] *= tk; gy[k] *= tk; gz[k] *= tk; gt[k] *= tk;
    }
  }
  for (int q = q0 + gl; q < q1; q += G) {
    const int2 fj = lfj[q];
    const int f = fj.x;
    const unsigned char ff = fflag[f];
    if (!(ff & FF_ACTIVE) || (ff & (FF_BND1 | FF_BND2))) continue;
    const bool own = fj.y >= 0;
    const double tj = tlast[own ? fj.y : ~fj.y];
    const double dtI = t_global - (own ? ti : tj), dtJ = t_global - (own ? tj : ti);
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
    const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1, const unsigned char *FVM_RESTRICT fflag,
    const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT tlast,
    const R *FVM_RESTRICT Wrec, R *FVM_RESTRICT tau, R *FVM_RESTRICT fst, const int *FVM_RESTRICT perm,
    const R *FVM_RESTRICT mnmx, const unsigned char *FVM_RESTRICT mz, const R *FVM_RESTRICT lld) {
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
__global__ void __launch_bounds__(128, MINB) k_limiter_st(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1, const unsigned char *FVM_RESTRICT fflag,
    const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT tlast,
    const R *FVM_RESTRICT Wrec, R *FVM_RESTRICT tau, R *FVM_RESTRICT fst, const int *FVM_RESTRICT perm,
    const R *FVM_RESTRICT mnmx, const unsigned char *FVM_RESTRICT mz, int only_all, const R *FVM_RESTRICT lld) {
  constexpr int CST = limiter_cst<KH>();
  extern __shared__ __align__(16) unsigned char lsm[];
  __shared__ int soff[CST + 1];
  if (only_all && S->iscal[1] != n) return;
  const double t_global = S->t_global;
  const bool reuse = FVM_REUSE_MINMAX && S->mnmx_ok && S->iscal[1] == n;
  // one cell block per block, or (a grid smaller than the cell blocks, as
  // partial steps launch it, where it usually has nothing to do) a loop over
  // them; a block's threads meet at the block's barriers in every pass
  const int ncb = (n + CST - 1) / CST;
  for (int cb = blockIdx.x; cb < ncb; cb += gridDim.x) {
    if (cb != (int)blockIdx.x) __syncthreads();  // the previous pass is done with the staging
    limiter_st_block<R, KH>(cb, n, reuse, t_global, soff, lsm, off, lnk, lfj, s12, geo, dr1, fflag, act, tlast,
                            Wrec, tau, fst, perm, mnmx, mz, lld);
  }
}
template <typename R, int KH, int MINB>
__device__ __forceinline__ void limiter_dev(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1, const unsigned char *FVM_RESTRICT fflag,
    const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT tlast,
    const R *FVM_RESTRICT Wrec, R *FVM_RESTRICT tau, R *FVM_RESTRICT fst, const int *FVM_RESTRICT perm,
    const R *FVM_RESTRICT mnmx, const unsigned char *FVM_RESTRICT mz, const int *FVM_RESTRICT clist,
    int skip_if_all, const R *FVM_RESTRICT lld, int gt0_, int gnt_) {
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
  for (long long t = (long long)gt0_; t < cnt;
       t += (long long)gnt_) {
    const int u = (int)(t / TPC);
    limiter_thread<R, KH>(lst ? clist[u] : perm[u], (int)(t % TPC) * KH, reuse, t_global, off, lnk, lfj, s12, geo,
                          dr1, fflag, act, tlast, Wrec, tau, fst, mnmx, mz, lld);
  }
}
template <typename R, int KH, int MINB>
__global__ void __launch_bounds__(128, MINB) k_limiter(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1, const unsigned char *FVM_RESTRICT fflag,
    const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT tlast,
    const R *FVM_RESTRICT Wrec, R *FVM_RESTRICT tau, R *FVM_RESTRICT fst, const int *FVM_RESTRICT perm,
    const R *FVM_RESTRICT mnmx, const unsigned char *FVM_RESTRICT mz, const int *FVM_RESTRICT clist,
    int skip_if_all, const R *FVM_RESTRICT lld) {
  limiter_dev<R, KH, MINB>(n, P, S, off, lnk, lfj, s12, geo, dr1, fflag, act, tlast, Wrec, tau, fst, perm, mnmx, mz, clist, skip_if_all, lld, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
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
__device__ __forceinline__ void corr_face(int f, int slot, double t_global, const Params &P, const Sched *FVM_RESTRICT S,
    const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
    const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT vel,
    const double *FVM_RESTRICT tlast, const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT fst,
    R *FVM_RESTRICT fcon, unsigned char *FVM_RESTRICT fcode, const LearnBuf &lb) {
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
__device__ __forceinline__ void corr_flux_dev(int nf, Params P, const Sched *FVM_RESTRICT S,
    const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
    const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT vel,
    const double *FVM_RESTRICT tlast, const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT fst,
    R *FVM_RESTRICT fcon, unsigned char *FVM_RESTRICT fcode, LearnBuf lb, const int *FVM_RESTRICT flist,
    int use_list, int gt0_, int gnt_) {
  const double t_global = S->t_global;
  const int t = gt0_;
  if (MODE == LM_FINISH) {  // one deferred face per thread
    if (t >= *lb.count) return;
    corr_face<R, MODE>(lb.gface[t], t, t_global, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec, fst, fcon, fcode, lb);
  } else if (use_list) {  // the active faces (the others were coded F_OFF with the flags)
    const int na = S->iscal[3];
    for (int u = t; u < na; u += gnt_)  // the list is built only when some face is inactive
      corr_face<R, MODE>(na != nf ? flist[u] : u, -1, t_global, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec,
                         fst, fcon, fcode, lb);
  } else if (t < nf) {
    corr_face<R, MODE>(t, -1, t_global, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec, fst, fcon, fcode, lb);
  }
}
template <typename R, int MODE, int MB = FVM_FLUX_MINB(R)>
__global__ void __launch_bounds__(128, MB) k_corr_flux(int nf, Params P, const Sched *FVM_RESTRICT S,
    const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
    const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT vel,
    const double *FVM_RESTRICT tlast, const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT fst,
    R *FVM_RESTRICT fcon, unsigned char *FVM_RESTRICT fcode, LearnBuf lb, const int *FVM_RESTRICT flist,
    int use_list) {
  corr_flux_dev<R, MODE>(nf, P, S, s12, geo, dr1, fflag, bnd, vel, tlast, Wrec, fst, fcon, fcode, lb, flist, use_list, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
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
__device__ __forceinline__ void gather_contrib(int c, int q0, int q1, const int2 *FVM_RESTRICT lfj,
                                               const R *FVM_RESTRICT fcon,
                                               const unsigned char *FVM_RESTRICT fcode, bool skipj_allowed,
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

// The same sums with G consecutive lanes per cell (G a power of two, gmask
// the group's lanes, gl this lane's index in it): lane gl loads the records
// of links q0 + gl, q0 + gl + G, ..., and every lane of the group adds all
// the records in link order, each taken by shuffle from the lane that
// loaded it, with the operations of gather_contrib: the sums are its bits,
// and a cell's walk is q1 - q0 over G loads deep instead of q1 - q0.
template <typename R, int G>
__device__ __forceinline__ void gather_contrib_group(int q0, int q1, const int2 *FVM_RESTRICT lfj,
                                                     const R *FVM_RESTRICT fcon,
                                                     const unsigned char *FVM_RESTRICT fcode, bool skipj_allowed,
                                                     int gl, unsigned gmask, double *s) {
  constexpr bool kahan = sizeof(R) == 4;
  double comp[14];
#pragma unroll
  for (int k = 0; k < 14; k++) { s[k] = 0.0; comp[k] = 0.0; }
  for (int base = q0; base < q1; base += G) {
    const int q = base + gl;
    R vr[14];  // the record as stored; the side and use bits travel with it
    int info = 0;
    if (q < q1) {
      const int2 fj = lfj[q];
      const int f = fj.x;
      load_n<R, 14>(fcon + 14 * (size_t)f, vr);
      const unsigned char code = fcode[f];
      const bool is_i = (fj.y >= 0) != ((code & F_SWAP) != 0);
      const bool use = !(code & F_OFF) && !(!is_i && skipj_allowed && (code & F_SKIPJ));
      info = (is_i ? 1 : 0) | (use ? 2 : 0);
    } else {
#pragma unroll
      for (int k = 0; k < 14; k++) vr[k] = R(0);
    }
    const int m = min(G, q1 - base);
    for (int j = 0; j < m; j++) {
      const int ij = __shfl_sync(gmask, info, j, G);
      const bool is_i = ij & 1, use = (ij & 2) != 0;
      const double wu = is_i ? -1.0 : 1.0;
#pragma unroll
      for (int k = 0; k < 14; k++) {
        const double v = double(__shfl_sync(gmask, vr[k], j, G));
        if (kahan) {
          const double term = ((k < NF) == is_i) ? -v : v;
          const double y = term - comp[k];
          const double t = s[k] + y;
          comp[k] = use ? (t - s[k]) - y : comp[k];
          s[k] = use ? t : s[k];
        } else {
          // fma(+-1, use ? v : 0, s) of gather_contrib: the product is exact
          s[k] = s[k] + (k < NF ? wu : -wu) * (use ? v : 0.0);
        }
      }
    }
  }
}

// ---- compute_update cell pass (MPI/compute_update.cpp:274-498) -----------
// The cell's update from its summed face contributions s (ac: its act
// flags, active or local neighbour).
template <typename R>
__device__ __forceinline__ void corr_cell_finish(int c, unsigned char ac, const double *s, double t_global,
    const Params &P, const double *FVM_RESTRICT cvol, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast, double *FVM_RESTRICT volp,
    const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT tau,
    double *FVM_RESTRICT U, double *FVM_RESTRICT dU, double *FVM_RESTRICT stepdU,
    unsigned long long *FVM_RESTRICT counters, float *FVM_RESTRICT divb) {
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
    const double l_min = P.hcell[c];
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

template <typename R>
__device__ __forceinline__ void corr_cell_body(int c, double t_global, const Params &P,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast, double *FVM_RESTRICT volp,
    const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT tau,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    double *FVM_RESTRICT U, double *FVM_RESTRICT dU, double *FVM_RESTRICT stepdU,
    unsigned long long *FVM_RESTRICT counters, float *FVM_RESTRICT divb) {
  const unsigned char ac = act[c];
  if (!(ac & (A_ACTIVE | A_LNGB))) return;
  double s[14];
  gather_contrib<R>(c, off[c], off[c + 1], lfj, fcon, fcode, true, s);
  corr_cell_finish<R>(c, ac, s, t_global, P, cvol, bnd, pos, tlast, volp, Wrec, tau, U, dU, stepdU, counters, divb);
}

// The same with G lanes per cell (gather_contrib_group; the group's first
// lane finishes the cell).
template <typename R, int G>
__device__ __forceinline__ void corr_cell_group(int c, int gl, unsigned gmask, double t_global, const Params &P,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast, double *FVM_RESTRICT volp,
    const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT tau,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    double *FVM_RESTRICT U, double *FVM_RESTRICT dU, double *FVM_RESTRICT stepdU,
    unsigned long long *FVM_RESTRICT counters, float *FVM_RESTRICT divb) {
  const unsigned char ac = act[c];
  if (!(ac & (A_ACTIVE | A_LNGB))) return;
  double s[14];
  gather_contrib_group<R, G>(off[c], off[c + 1], lfj, fcon, fcode, true, gl, gmask, s);
  if (gl == 0)
    corr_cell_finish<R>(c, ac, s, t_global, P, cvol, bnd, pos, tlast, volp, Wrec, tau, U, dU, stepdU, counters,
                        divb);
}

// One thread per cell; in partial steps a fixed grid strides over the
// involved-cell list (clist, count ninv) instead of every cell.
template <typename R>
__device__ __forceinline__ void corr_cell_dev(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast, double *FVM_RESTRICT volp,
    const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT tau,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    double *FVM_RESTRICT U, double *FVM_RESTRICT dU, double *FVM_RESTRICT stepdU,
    unsigned long long *FVM_RESTRICT counters, const int *FVM_RESTRICT perm, float *FVM_RESTRICT divb,
    const int *FVM_RESTRICT clist, int gt0_, int gnt_) {
  const double t_global = S->t_global;
  const int cnt = clist ? S->ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = gt0_; t < cnt; t += gnt_)
    corr_cell_body<R>(lst ? clist[t] : perm[t], t_global, P, off, lfj, cvol, act, bnd, pos, tlast, volp, Wrec, tau,
                      fcon, fcode, U, dU, stepdU, counters, divb);
}
template <typename R>
__global__ void __launch_bounds__(128) k_corr_cell(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast, double *FVM_RESTRICT volp,
    const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT tau,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    double *FVM_RESTRICT U, double *FVM_RESTRICT dU, double *FVM_RESTRICT stepdU,
    unsigned long long *FVM_RESTRICT counters, const int *FVM_RESTRICT perm, float *FVM_RESTRICT divb,
    const int *FVM_RESTRICT clist) {
  corr_cell_dev<R>(n, P, S, off, lfj, s12, cvol, act, bnd, pos, tlast, volp, Wrec, tau, fcon, fcode, U, dU, stepdU, counters, perm, divb, clist, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
// The same for global steps, with more resident blocks.
template <typename R>
__global__ void __launch_bounds__(128, FVM_CORR_CELL_MINB(R)) k_corr_cell_g(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast, double *FVM_RESTRICT volp,
    const R *FVM_RESTRICT Wrec, const R *FVM_RESTRICT tau,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    double *FVM_RESTRICT U, double *FVM_RESTRICT dU, double *FVM_RESTRICT stepdU,
    unsigned long long *FVM_RESTRICT counters, const int *FVM_RESTRICT perm, float *FVM_RESTRICT divb,
    const int *FVM_RESTRICT clist) {
  corr_cell_dev<R>(n, P, S, off, lfj, s12, cvol, act, bnd, pos, tlast, volp, Wrec, tau, fcon, fcode, U, dU, stepdU, counters, perm, divb, clist, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---- compute_pvel (MPI/compute_pvel.cpp:5-52) -----------------------------
__device__ __forceinline__ void pvel_body(int i, const Params &P, const unsigned char *FVM_RESTRICT act,
                       const int *FVM_RESTRICT bnd,
                       const double *FVM_RESTRICT U, const double *FVM_RESTRICT volp,
                       const double *FVM_RESTRICT cvol, const double *FVM_RESTRICT ccen,
                       const double *FVM_RESTRICT pos, double *FVM_RESTRICT vel) {
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
__device__ __forceinline__ void pvel_dev(int n, Params P, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
                       const double *FVM_RESTRICT U, const double *FVM_RESTRICT volp,
                       const double *FVM_RESTRICT cvol, const double *FVM_RESTRICT ccen,
                       const double *FVM_RESTRICT pos, double *FVM_RESTRICT vel, const int *FVM_RESTRICT clist,
                       const int *FVM_RESTRICT ninv, int gt0_, int gnt_) {
  const int cnt = clist ? *ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = gt0_; t < cnt; t += gnt_)
    pvel_body(lst ? clist[t] : t, P, act, bnd, U, volp, cvol, ccen, pos, vel);
}
__global__ void k_pvel(int n, Params P, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
                       const double *FVM_RESTRICT U, const double *FVM_RESTRICT volp,
                       const double *FVM_RESTRICT cvol, const double *FVM_RESTRICT ccen,
                       const double *FVM_RESTRICT pos, double *FVM_RESTRICT vel, const int *FVM_RESTRICT clist,
                       const int *FVM_RESTRICT ninv) {
  pvel_dev(n, P, act, bnd, U, volp, cvol, ccen, pos, vel, clist, ninv, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---- compute_timestep(i) (MPI/compute_timestep.cpp:6-51) ------------------
// The face minimum min_f h / x_f is taken as h / max_f x_f: h > 0 and a
// rounded quotient never increases with its divisor, so both give the same
// double, with one division instead of one per face.  With G > 1 lanes per
// cell (gl this lane's index in its group, gmask the group's lanes) every
// lane computes the cell's own terms, the faces are split among the lanes
// and their maximum is reduced by shuffles: a maximum does not depend on the
// order, so every lane gets the double one lane would.
template <int G = 1>
__device__ double cell_timestep(const Params &P, int i, bool with_faces, const int *off, const int2 *lfj,
                                const int *bnd, const double *U, const double *volp, const double *vel, int gl = 0,
                                unsigned gmask = 0xffffffffu) {
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
  const double h = P.hcell[i];  // volp is the cell's volume
  double dti = h / (csi + vrel + 1.0 / FVM_HUGE);
  if (with_faces) {
    const double fac = b ? 0.0 : 1.0;
    double xmax = 0.0;
    const int q0 = off[i], q1 = off[i + 1];
    for (int q = q0 + gl; q < q1; q += G) {
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
    for (int o = G / 2; o > 0; o >>= 1) xmax = smax(xmax, __shfl_xor_sync(gmask, xmax, o, G));
    if (q1 > q0) dti = smin(dti, h / xmax);
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

// compute_timesteps(false) first loops (MPI/compute_timestep.cpp:78-96) with
// G lanes per cell (cell_timestep's faces split among them), over the
// involved-cell list or every cell; the group's first lane writes the cell's
// dt and takes part in the global minimum, reduced per warp before one
// atomic per warp.
template <int G>
__device__ __forceinline__ void timestep_group(Params P, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                           const unsigned char *FVM_RESTRICT act,
                           const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT U,
                           const double *FVM_RESTRICT volp, const double *FVM_RESTRICT vel,
                           const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast,
                           const double *FVM_RESTRICT tend, double *FVM_RESTRICT dtl,
                           double *FVM_RESTRICT dmin, const int *FVM_RESTRICT clist, int ninv, int gl,
                           unsigned gmask, int g0, int gn, int n = 0) {
  // clist and its count ninv, or (clist null) every one of the n cells
  double vmin = FVM_HUGE;
  const int cnt = clist ? ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t_ = g0; t_ < cnt; t_ += gn) {
    const int i = lst ? clist[t_] : t_;
    const unsigned char a = act[i];
    if (!(a & (A_ACTIVE | A_LNGB))) {
      if (gl == 0) dtl[i] = FVM_HUGE;
    } else if (!(a & A_ACTIVE)) {
      if (gl == 0) dtl[i] = (tend[i] - tlast[i]) * (bnd[i] != NO_BOUNDARY ? -1.0 : 1.0);
    } else {
      const double dti = smin(extra_timestep(P, i, bnd, pos, vel),
                              cell_timestep<G>(P, i, true, off, lfj, bnd, U, volp, vel, gl, gmask));
      if (gl == 0) {
        if (!P.halo || !P.halo[i]) vmin = smin(vmin, dti);
        dtl[i] = bnd[i] != NO_BOUNDARY ? -1.0 * dti : dti;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) vmin = smin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0 && vmin < FVM_HUGE) atomic_min_pos(dmin, vmin);
}

__global__ void k_timestep(int n, Params P, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                           const unsigned char *FVM_RESTRICT act,
                           const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT U,
                           const double *FVM_RESTRICT volp, const double *FVM_RESTRICT vel,
                           const double *FVM_RESTRICT pos, const double *FVM_RESTRICT tlast,
                           const double *FVM_RESTRICT tend, double *FVM_RESTRICT dtl,
                           double *FVM_RESTRICT dmin, const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv) {
  // one thread per cell: every lane of a group would repeat the cell's own
  // terms (a cube root among them), and on a full step that costs more than
  // the shorter face walk gains (0.26 -> 0.69 ms on the 128^3 blast)
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
  timestep_group<1>(P, off, lfj, act, bnd, U, volp, vel, pos, tlast, tend, dtl, dmin, clist, clist ? *ninv : 0, 0,
                    0xffffffffu, gt, gn, n);
}

// dt >= 8 dt_min halving (MPI/compute_timestep.cpp:103-104)
__device__ __forceinline__ void halve_dev(int n, const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT dmin,
                        double *FVM_RESTRICT dtl, const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv, int gt0_, int gnt_) {
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = gt0_; t_ < cnt_; t_ += gnt_) {
    const int i = lst ? clist[t_] : t_;
    if ((act[i] & A_ACTIVE) && dtl[i] >= 8.0 * dmin[0]) dtl[i] *= 0.5;
  }
}
__global__ void k_halve(int n, const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT dmin,
                        double *FVM_RESTRICT dtl, const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv) {
  halve_dev(n, act, dmin, dtl, clist, ninv, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
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
// The marks with G lanes per site, over the involved-cell list or every
// cell: the faces split among the lanes (the marks do not depend on the
// order), the site's own marks and count by the group's first lane.  Called
// by every thread of the block.
template <int G>
__device__ __forceinline__ void adjust_mark_group(const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                              const unsigned char *FVM_RESTRICT act,
                              const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT dtl,
                              unsigned char *FVM_RESTRICT hash, int *FVM_RESTRICT ndirty,
                              unsigned char *FVM_RESTRICT site, unsigned char *FVM_RESTRICT work,
                              const int *FVM_RESTRICT clist, int ninv, int gl, unsigned gmask, int g0, int gn,
                              int n = 0) {
  int ndirty_t = 0;
  const int cnt = clist ? ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t_ = g0; t_ < cnt; t_ += gn) {
    const int i = lst ? clist[t_] : t_;
    if (!(act[i] & A_ACTIVE) || bnd[i] != NO_BOUNDARY) continue;
    bool dirty = false;
    const double di = dtl[i];
    for (int q = off[i] + gl; q < off[i + 1]; q += G) {
      const int2 fj = lfj[q];
      const int j = fj.y >= 0 ? fj.y : ~fj.y;
      const double dj = dtl[j];
      if (dj < 0.0) continue;
      hash[j] = 1;
      if (2.0 * dj < di || 2.0 * di < dj) {
        dirty = true;
        work[j] = 1;
      }
    }
    dirty = __any_sync(gmask, dirty);
    if (gl == 0) {
      site[i] = 1;
      if (dirty) { work[i] = 1; ndirty_t++; }
    }
  }
  __shared__ int bsum;
  if (threadIdx.x == 0) bsum = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) ndirty_t += __shfl_xor_sync(0xffffffffu, ndirty_t, o);
  if ((threadIdx.x & 31) == 0 && ndirty_t) atomicAdd(&bsum, ndirty_t);
  __syncthreads();
  if (threadIdx.x == 0 && bsum) atomicAdd(ndirty, bsum);
}

__global__ void k_adjust_mark(int n, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                              const unsigned char *FVM_RESTRICT act,
                              const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT dtl,
                              unsigned char *FVM_RESTRICT hash, int *FVM_RESTRICT ndirty,
                              unsigned char *FVM_RESTRICT site, unsigned char *FVM_RESTRICT work,
                              const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv) {
  // eight lanes per site (adjust_mark_group)
  constexpr int G = 8;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
  const unsigned gmask = ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
  adjust_mark_group<G>(off, lfj, act, bnd, dtl, hash, ndirty, site, work, clist, clist ? *ninv : 0,
                       gt & (G - 1), gmask, gt / G, gn / G, n);
}

// Order-preserving compaction of flagged cells: per-block counts, one-block
// exclusive scan of the counts, then per-block placement.
constexpr int CB = 1024;
__global__ void k_count_flags(int n, const unsigned char *FVM_RESTRICT flag, int *FVM_RESTRICT bcount) {
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
__global__ void k_scan_counts(int nb, int *FVM_RESTRICT bcount, int *FVM_RESTRICT total) {
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
__global__ void k_place_flags(int n, const unsigned char *FVM_RESTRICT flag, const int *FVM_RESTRICT boff,
                              int *FVM_RESTRICT list) {
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
__global__ void k_place_faces(int nf, const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT nactive,
                              const int *FVM_RESTRICT boff, int *FVM_RESTRICT list) {
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
__global__ void k_count_cells(int n, const unsigned char *FVM_RESTRICT act, int *FVM_RESTRICT bcount) {
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
__global__ void k_place_cells(int n, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT boff,
                              int *FVM_RESTRICT list) {
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

// The sweep itself, on one thread.
__device__ __forceinline__ void adjust_seq_dev(const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk,
                                               const int2 *FVM_RESTRICT s12, const int *FVM_RESTRICT alist,
                                               const int *FVM_RESTRICT nsite, const int *FVM_RESTRICT ndirty,
                                               double *FVM_RESTRICT dtl) {
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

__global__ void k_adjust_seq(const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk,
                             const int2 *FVM_RESTRICT s12, const int *FVM_RESTRICT alist,
                             const int *FVM_RESTRICT nsite, const int *FVM_RESTRICT ndirty,
                             double *FVM_RESTRICT dtl) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  adjust_seq_dev(off, lnk, s12, alist, nsite, ndirty, dtl);
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

// G consecutive lanes per cell (the link entries are independent of one
// another), gt0_ and gnt_ in lanes.
template <int G = 1>
__device__ __forceinline__ void adjust_init_dev(int n, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                              const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT ndirty,
                              const double *FVM_RESTRICT dtl, double *FVM_RESTRICT dt0, double *FVM_RESTRICT rdv,
                              double *FVM_RESTRICT wrv, int *FVM_RESTRICT aflag, const int *FVM_RESTRICT clist,
                              const int *FVM_RESTRICT ninv, int gt0_, int gnt_) {
  if (*ndirty == 0) return;  // every pair is within a factor 2: nothing changes
  if (gt0_ == 0) aflag[2] = 1;  // replay 0 runs
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  const int gl = gt0_ % G;
  for (int t_ = gt0_ / G; t_ < cnt_; t_ += gnt_ / G) {
    const int u = lst ? clist[t_] : t_;
    if (!(act[u] & (A_ACTIVE | A_LNGB))) continue;
    const double du = dtl[u];
    if (gl == 0) dt0[u] = du;
    for (int q = off[u] + gl; q < off[u + 1]; q += G) {
      const int v = lfj_nb(lfj[q]);
      rdv[q] = (act[v] & (A_ACTIVE | A_LNGB)) ? dtl[v] : du;
      wrv[q] = du;
    }
  }
}
__global__ void k_adjust_init(int n, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                              const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT ndirty,
                              const double *FVM_RESTRICT dtl, double *FVM_RESTRICT dt0, double *FVM_RESTRICT rdv,
                              double *FVM_RESTRICT wrv, int *FVM_RESTRICT aflag, const int *FVM_RESTRICT clist,
                              const int *FVM_RESTRICT ninv) {
  adjust_init_dev<8>(n, off, lfj, act, ndirty, dtl, dt0, rdv, wrv, aflag, clist, ninv,
                     blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__device__ __forceinline__ void adjust_replay_dev(int n, int kparam, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                                const int *FVM_RESTRICT lsort, const int *FVM_RESTRICT lpart,
                                const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT dt0,
                                double *FVM_RESTRICT rdv, double *FVM_RESTRICT wrv, double *FVM_RESTRICT dtl,
                                int *FVM_RESTRICT aflag, unsigned char *FVM_RESTRICT work, int kdev, int gt0_, int gnt_,
                                const int *FVM_RESTRICT ulist = nullptr, int ucount = 0) {
  // replay index: the launch's, or (in a captured step) aflag[7], which
  // k_adjust_next advances between replays
  const int k = kdev ? aflag[7] : kparam;
  const int t0 = gt0_;
  if (aflag[5]) return;
  if (aflag[(k + 2) % 3] == 0) {  // the previous replay changed nothing (or none was needed)
    if (t0 == 0) aflag[5] = 1;
    return;
  }
  if (t0 == 0) { aflag[(k + 1) % 3] = 0; aflag[3] += 1; }
  bool changed = false;
  unsigned char *cur = work + (size_t)(k & 1) * n, *nxt = work + (size_t)((k + 1) & 1) * n;
  // every cell (grid-stride: a settled replay costs one launch), or only the
  // cells of ulist, which then holds every cell a work list can name
  const int ucnt = ulist ? ucount : n;
  for (int tu = t0; tu < ucnt; tu += gnt_) {
    const int u = ulist ? ulist[tu] : tu;
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
__global__ void k_adjust_replay(int n, int kparam, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                                const int *FVM_RESTRICT lsort, const int *FVM_RESTRICT lpart,
                                const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT dt0,
                                double *FVM_RESTRICT rdv, double *FVM_RESTRICT wrv, double *FVM_RESTRICT dtl,
                                int *FVM_RESTRICT aflag, unsigned char *FVM_RESTRICT work, int kdev,
                                const int *FVM_RESTRICT ulist, const int *FVM_RESTRICT ucount) {
  adjust_replay_dev(n, kparam, off, lfj, lsort, lpart, act, dt0, rdv, wrv, dtl, aflag, work, kdev,
                    blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, ulist, ulist ? *ucount : 0);
}

// A partial step's adjust_timesteps work arrays, cleared for its involved
// cells only: every mark, work list and replay write of the step lands on
// one of them, and every reader walks them only (the replays through their
// list, the site compaction below).
__global__ void k_adjust_clear(int n, const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv,
                               unsigned char *FVM_RESTRICT hash, unsigned char *FVM_RESTRICT act0,
                               unsigned char *FVM_RESTRICT work) {
  const int cnt = *ninv;
  const bool lst = cnt != n;  // every cell involved: the list is the identity
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
    const int i = lst ? clist[t] : t;
    hash[i] = 0;
    act0[i] = 0;
    work[i] = 0;
    work[(size_t)n + i] = 0;
  }
}

// The active non-boundary sites (act0) in ascending order from the ascending
// involved-cell list, in two launches of SITE_BLOCKS blocks over contiguous
// chunks of it: k_site_count counts each chunk's sites, k_site_place writes
// them after the counts of the chunks before (alist, count in *nsites).
// Enough blocks that a chunk of a step with every cell involved is a few
// rounds of the block.
constexpr int SITE_BLOCKS = 512;
__device__ __forceinline__ void site_chunk(int cnt, int &t0, int &t1) {
  const int C = (cnt + SITE_BLOCKS - 1) / SITE_BLOCKS;
  t0 = blockIdx.x * C;
  t1 = min(cnt, t0 + C);
}
__global__ void __launch_bounds__(256) k_site_count(int n, const int *FVM_RESTRICT clist,
                                                    const int *FVM_RESTRICT ninv,
                                                    const unsigned char *FVM_RESTRICT act0, int *FVM_RESTRICT bcnt) {
  __shared__ int wsum[8];
  const int cnt = *ninv;
  const bool lst = cnt != n;
  int t0, t1;
  site_chunk(cnt, t0, t1);
  int c = 0;
  for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) c += act0[lst ? clist[t] : t] != 0;
  const int tot = block_sum(c, wsum);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = tot;
}
__global__ void __launch_bounds__(256) k_site_place(int n, const int *FVM_RESTRICT clist,
                                                    const int *FVM_RESTRICT ninv,
                                                    const unsigned char *FVM_RESTRICT act0,
                                                    const int *FVM_RESTRICT bcnt, int *FVM_RESTRICT alist,
                                                    int *FVM_RESTRICT nsites) {
  __shared__ int wsum[8], base;
  if (threadIdx.x < 32) {
    int before = 0, all = 0;
    for (int b = threadIdx.x; b < SITE_BLOCKS; b += 32) {
      const int v = bcnt[b];
      all += v;
      before += b < (int)blockIdx.x ? v : 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
      before += __shfl_xor_sync(0xffffffffu, before, o);
      all += __shfl_xor_sync(0xffffffffu, all, o);
    }
    if (threadIdx.x == 0) {
      base = before;
      if (blockIdx.x == 0) *nsites = all;
    }
  }
  __syncthreads();
  const int cnt = *ninv;
  const bool lst = cnt != n;
  int t0, t1;
  site_chunk(cnt, t0, t1);
  // the chunk in rounds of blockDim entries, each placed by a block scan
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int r0 = t0; r0 < t1; r0 += blockDim.x) {
    const int t = r0 + threadIdx.x;
    const int i = t < t1 ? (lst ? clist[t] : t) : -1;
    const bool f = i >= 0 && act0[i] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    int o = base;
    for (int w = 0; w < wid; w++) o += wsum[w];
    if (f) alist[o + __popc(bal & ((1u << lane) - 1u))] = i;
    __syncthreads();
    if (threadIdx.x == 0)
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) base += wsum[w];
    __syncthreads();
  }
}

// In a captured step the replays run as the body of a conditional WHILE
// node: after replay k this single thread stops the loop once replay k
// changed nothing (settled) or ADJ_ITERS replays have run, and advances k.
__global__ void k_adjust_next(int *FVM_RESTRICT aflag, cudaGraphConditionalHandle loop) {
  const int k = aflag[7];
  bool stop = aflag[5] != 0;
  if (aflag[k % 3] == 0) { aflag[5] = 1; stop = true; }
  if (k + 1 >= ADJ_ITERS) stop = true;
  aflag[7] = k + 1;
  cudaGraphSetConditional(loop, stop ? 0u : 1u);
}

// Not settled after ADJ_ITERS replays: restore the initial dt for the
// sequential sweep.
__device__ __forceinline__ void adjust_restore_dev(int n, const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT dt0,
                                 double *FVM_RESTRICT dtl, int *FVM_RESTRICT aflag, int *FVM_RESTRICT stats,
                                 const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv, int gt0_, int gnt_) {
  const bool fallback = !aflag[5] && aflag[(ADJ_ITERS - 1) % 3] != 0;
  const bool first = gt0_ == 0;
  if (first) { stats[0] = aflag[3]; stats[1] = fallback ? 1 : 0; }
  if (!fallback) return;
  if (first) aflag[4] = 1;
  const int cnt_ = clist ? *ninv : n;
  const bool lst = clist && cnt_ != n;  // every cell involved: the list is the identity
  for (int t_ = gt0_; t_ < cnt_; t_ += gnt_) {
    const int u = lst ? clist[t_] : t_;
    if (act[u] & (A_ACTIVE | A_LNGB)) dtl[u] = dt0[u];
  }
}
__global__ void k_adjust_restore(int n, const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT dt0,
                                 double *FVM_RESTRICT dtl, int *FVM_RESTRICT aflag, int *FVM_RESTRICT stats,
                                 const int *FVM_RESTRICT clist, const int *FVM_RESTRICT ninv) {
  adjust_restore_dev(n, act, dt0, dtl, aflag, stats, clist, ninv, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// rung assignment and inactive-neighbour promotion (MPI/compute_timestep.cpp
// :144-199) fused with collect_results (MPI/distribute_work.cpp:676-713) and
// the tlast/tend update of correct() (set_problem.cpp generic hook)
template <typename R>
__device__ __forceinline__ void rungs_body(int i, double t_global, int min_rung, const Params &P, int shared,
                        const unsigned char *FVM_RESTRICT act, const unsigned char *FVM_RESTRICT hash,
                        const double *FVM_RESTRICT dtl, const double *FVM_RESTRICT dmin,
                        int *FVM_RESTRICT rung, double *FVM_RESTRICT tlast, double *FVM_RESTRICT tend,
                        R *FVM_RESTRICT Wrec, int *FVM_RESTRICT iscal, const double *FVM_RESTRICT vel,
                        double *FVM_RESTRICT opos, double *FVM_RESTRICT ovel) {
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
__device__ __forceinline__ void rungs_dev(int n, Params P, const Sched *FVM_RESTRICT S, int shared,
                        const unsigned char *FVM_RESTRICT act, const unsigned char *FVM_RESTRICT hash,
                        const double *FVM_RESTRICT dtl, const double *FVM_RESTRICT dmin,
                        int *FVM_RESTRICT rung, double *FVM_RESTRICT tlast, double *FVM_RESTRICT tend,
                        R *FVM_RESTRICT Wrec, int *FVM_RESTRICT iscal, const double *FVM_RESTRICT vel,
                        double *FVM_RESTRICT opos, double *FVM_RESTRICT ovel, const int *FVM_RESTRICT clist, int gt0_, int gnt_) {
  const double t_global = S->t_global;
  const int min_rung = S->min_rung;
  const int cnt = clist ? S->ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = gt0_; t < cnt; t += gnt_)
    rungs_body<R>(lst ? clist[t] : t, t_global, min_rung, P, shared, act, hash, dtl, dmin, rung, tlast, tend, Wrec,
                  iscal, vel, opos, ovel);
}
template <typename R>
__global__ void k_rungs(int n, Params P, const Sched *FVM_RESTRICT S, int shared,
                        const unsigned char *FVM_RESTRICT act, const unsigned char *FVM_RESTRICT hash,
                        const double *FVM_RESTRICT dtl, const double *FVM_RESTRICT dmin,
                        int *FVM_RESTRICT rung, double *FVM_RESTRICT tlast, double *FVM_RESTRICT tend,
                        R *FVM_RESTRICT Wrec, int *FVM_RESTRICT iscal, const double *FVM_RESTRICT vel,
                        double *FVM_RESTRICT opos, double *FVM_RESTRICT ovel, const int *FVM_RESTRICT clist) {
  rungs_dev<R>(n, P, S, shared, act, hash, dtl, dmin, rung, tlast, tend, Wrec, iscal, vel, opos, ovel, clist, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// distribute_fluid_update_data: primitives of the updated state
template <typename R>
__device__ __forceinline__ void wst_body(int i, const unsigned char *FVM_RESTRICT act,
                                         const double *FVM_RESTRICT U, const double *FVM_RESTRICT volp,
                                         R *FVM_RESTRICT Wst) {
  if (!(act[i] & (A_ACTIVE | A_LNGB))) return;
  double u[NF], W[NF];
  load_n<double, NF>(U + 10 * (size_t)i, u);
  to_primitive(u, volp[i], W);
  R w[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) w[k] = R(W[k]);
  store_n<R, NF>(Wst + 10 * (size_t)i, w);
}
template <typename R>
__device__ __forceinline__ void wst_dev(int n, const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT U,
                      const double *FVM_RESTRICT volp, R *FVM_RESTRICT Wst, const int *FVM_RESTRICT clist,
                      const int *FVM_RESTRICT ninv, int gt0_, int gnt_) {
  const int cnt = clist ? *ninv : n;  // every cell, or in partial steps the involved-cell list
  const bool lst = clist && cnt != n;
  for (int t = gt0_; t < cnt; t += gnt_) wst_body<R>(lst ? clist[t] : t, act, U, volp, Wst);
}
template <typename R>
__global__ void k_wst(int n, const unsigned char *FVM_RESTRICT act, const double *FVM_RESTRICT U,
                      const double *FVM_RESTRICT volp, R *FVM_RESTRICT Wst, const int *FVM_RESTRICT clist,
                      const int *FVM_RESTRICT ninv) {
  wst_dev<R>(n, act, U, volp, Wst, clist, ninv, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---- compute_update0 face pass (MPI/compute_update.cpp:713-810) ----------
template <typename R, int MODE>
__device__ __forceinline__ void pred_face(int f, int slot, const Params &P,
    const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
    const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT vel, const R *FVM_RESTRICT Wst,
    R *FVM_RESTRICT fcon, unsigned char *FVM_RESTRICT fcode, const Sched *FVM_RESTRICT S, const int *FVM_RESTRICT rung,
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
__device__ __forceinline__ void pred_flux_dev(int nf, Params P,
    const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
    const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT vel, const R *FVM_RESTRICT Wst,
    R *FVM_RESTRICT fcon, unsigned char *FVM_RESTRICT fcode, const Sched *FVM_RESTRICT S, const int *FVM_RESTRICT rung,
    LearnBuf lb, const int *FVM_RESTRICT flist, int use_list, int gt0_, int gnt_) {
  const int t = gt0_;
  if (MODE == LM_FINISH) {
    if (t >= *lb.count) return;
    pred_face<R, MODE>(lb.gface[t], t, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb);
  } else if (use_list) {
    const int na = S->iscal[3];
    for (int u = t; u < na; u += gnt_)
      pred_face<R, MODE>(na != nf ? flist[u] : u, -1, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb);
  } else if (t < nf) {
    pred_face<R, MODE>(t, -1, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb);
  }
}
template <typename R, int MODE, int MB = FVM_FLUX_MINB(R)>
__global__ void __launch_bounds__(128, MB) k_pred_flux(int nf, Params P,
    const int2 *FVM_RESTRICT s12, const double4 *FVM_RESTRICT geo, const double4 *FVM_RESTRICT dr1,
    const unsigned char *FVM_RESTRICT fflag, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT vel, const R *FVM_RESTRICT Wst,
    R *FVM_RESTRICT fcon, unsigned char *FVM_RESTRICT fcode, const Sched *FVM_RESTRICT S, const int *FVM_RESTRICT rung,
    LearnBuf lb, const int *FVM_RESTRICT flist, int use_list) {
  pred_flux_dev<R, MODE>(nf, P, s12, geo, dr1, fflag, bnd, vel, Wst, fcon, fcode, S, rung, lb, flist, use_list, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---- compute_update0 cell pass + collect_reconstruction -------------------
// (MPI/compute_update.cpp:812-964; MPI/distribute_work.cpp:820-834)
// Writes the predicted time derivative t into the cell's Wrec and the
// cell's final rung/tend.  Arithmetic in double for both bulk types.
template <typename R>
__device__ __forceinline__ void pred_cell_finish(int c, const double *dot, double t_global, int min_rung,
    const Params &P, const double *FVM_RESTRICT cvol, const double *FVM_RESTRICT pos,
    const double *FVM_RESTRICT U, int *FVM_RESTRICT rung, double *FVM_RESTRICT tend, R *FVM_RESTRICT Wrec) {
  const double V = cvol[c];
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
    const double l_min = P.hcell[c];
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

template <typename R>
__device__ __forceinline__ void pred_cell_body(int c, double t_global, int min_rung, const Params &P,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT U,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    int *FVM_RESTRICT rung, double *FVM_RESTRICT tend, R *FVM_RESTRICT Wrec) {
  if (!(act[c] & A_ACTIVE) || bnd[c] != NO_BOUNDARY) return;
  double dot[14];
  gather_contrib<R>(c, off[c], off[c + 1], lfj, fcon, fcode, false, dot);
  pred_cell_finish<R>(c, dot, t_global, min_rung, P, cvol, pos, U, rung, tend, Wrec);
}

// The same with G lanes per cell (gather_contrib_group; the group's first
// lane finishes the cell).
template <typename R, int G>
__device__ __forceinline__ void pred_cell_group(int c, int gl, unsigned gmask, double t_global, int min_rung,
    const Params &P, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT U,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    int *FVM_RESTRICT rung, double *FVM_RESTRICT tend, R *FVM_RESTRICT Wrec) {
  if (!(act[c] & A_ACTIVE) || bnd[c] != NO_BOUNDARY) return;
  double dot[14];
  gather_contrib_group<R, G>(off[c], off[c + 1], lfj, fcon, fcode, false, gl, gmask, dot);
  if (gl == 0) pred_cell_finish<R>(c, dot, t_global, min_rung, P, cvol, pos, U, rung, tend, Wrec);
}

// One thread per cell; in partial steps a fixed grid strides over clist.
template <typename R>
__device__ __forceinline__ void pred_cell_dev(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT U,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    int *FVM_RESTRICT rung, double *FVM_RESTRICT tend, R *FVM_RESTRICT Wrec, const int *FVM_RESTRICT perm,
    const int *FVM_RESTRICT clist, int gt0_, int gnt_) {
  const double t_global = S->t_global;
  const int min_rung = S->min_rung;
  const int cnt = clist ? S->ninv : n;
  const bool lst = clist && cnt != n;  // every cell involved: the list is the identity
  for (int t = gt0_; t < cnt; t += gnt_)
    pred_cell_body<R>(lst ? clist[t] : perm[t], t_global, min_rung, P, off, lfj, cvol, act, bnd, pos, U, fcon,
                      fcode, rung, tend, Wrec);
}
template <typename R>
__global__ void __launch_bounds__(128) k_pred_cell(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT U,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    int *FVM_RESTRICT rung, double *FVM_RESTRICT tend, R *FVM_RESTRICT Wrec, const int *FVM_RESTRICT perm,
    const int *FVM_RESTRICT clist) {
  pred_cell_dev<R>(n, P, S, off, lfj, s12, cvol, act, bnd, pos, U, fcon, fcode, rung, tend, Wrec, perm, clist, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
// The same for global steps, with more resident blocks.
template <typename R>
__global__ void __launch_bounds__(128, FVM_PRED_CELL_MINB(R)) k_pred_cell_g(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj, const int2 *FVM_RESTRICT s12,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const double *FVM_RESTRICT pos, const double *FVM_RESTRICT U,
    const R *FVM_RESTRICT fcon, const unsigned char *FVM_RESTRICT fcode,
    int *FVM_RESTRICT rung, double *FVM_RESTRICT tend, R *FVM_RESTRICT Wrec, const int *FVM_RESTRICT perm,
    const int *FVM_RESTRICT clist) {
  pred_cell_dev<R>(n, P, S, off, lfj, s12, cvol, act, bnd, pos, U, fcon, fcode, rung, tend, Wrec, perm, clist, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ---- compute_reconstruction (MPI/compute_reconstruction.cpp:41-198) -------
// TPC threads per active cell, KH primitives each: Voronoi face gradient of
// the updated primitives, local limiter, density positivity rescale.
template <typename R, int KH>
__device__ __forceinline__ void recon_body(int c, int k0, const Params &P, const int *FVM_RESTRICT off,
    const int2 *FVM_RESTRICT lfj, const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act,
    const int *FVM_RESTRICT bnd, const R *FVM_RESTRICT Wst, const int *FVM_RESTRICT rung, R *FVM_RESTRICT Wrec,
    R *FVM_RESTRICT mnmx, unsigned char *FVM_RESTRICT mz, const R *FVM_RESTRICT lrw, const R *FVM_RESTRICT lrd,
    const unsigned char *FVM_RESTRICT bnb) {
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
__device__ __forceinline__ void recon_dev(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const R *FVM_RESTRICT Wst, const int *FVM_RESTRICT rung, R *FVM_RESTRICT Wrec, const int *FVM_RESTRICT perm,
    R *FVM_RESTRICT mnmx, unsigned char *FVM_RESTRICT mz, const R *FVM_RESTRICT lrw,
    const R *FVM_RESTRICT lrd, const int *FVM_RESTRICT clist, const unsigned char *FVM_RESTRICT bnb, int gt0_, int gnt_) {
  constexpr int TPC = 10 / KH;
  const long long cnt = (long long)TPC * (clist ? S->ninv : n);
  const bool lst = clist && S->ninv != n;  // every cell involved: the list is the identity
  for (long long t = (long long)gt0_; t < cnt;
       t += (long long)gnt_) {
    const int u = (int)(t / TPC);
    recon_body<R, KH>(lst ? clist[u] : perm[u], (int)(t % TPC) * KH, P, off, lfj, cvol, act, bnd, Wst, rung, Wrec,
                      mnmx, mz, lrw, lrd, bnb);
  }
}
template <typename R, int KH, int MINB>
__global__ void __launch_bounds__(128, MINB) k_recon(int n, Params P, const Sched *FVM_RESTRICT S,
    const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
    const double *FVM_RESTRICT cvol, const unsigned char *FVM_RESTRICT act, const int *FVM_RESTRICT bnd,
    const R *FVM_RESTRICT Wst, const int *FVM_RESTRICT rung, R *FVM_RESTRICT Wrec, const int *FVM_RESTRICT perm,
    R *FVM_RESTRICT mnmx, unsigned char *FVM_RESTRICT mz, const R *FVM_RESTRICT lrw,
    const R *FVM_RESTRICT lrd, const int *FVM_RESTRICT clist, const unsigned char *FVM_RESTRICT bnb) {
  recon_dev<R, KH, MINB>(n, P, S, off, lfj, cvol, act, bnd, Wst, rung, Wrec, perm, mnmx, mz, lrw, lrd, clist, bnb, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Per link (a cell's entry in its face list, i.e. one side of a face), in the
// order the cell walks its faces: the face id and the neighbour j, stored as
// ~j when the cell is s2.  The mesh is fixed while it is installed.
// Cells with a boundary neighbour, whose reconstruction is zero (the
// reference's face loop stops at such a neighbour,
// MPI/compute_reconstruction.cpp:103-106,121); boundary codes are fixed
// after the state is installed.
__global__ void k_bnd_neighbours(int n, const int *FVM_RESTRICT off, const int2 *FVM_RESTRICT lfj,
                                 const int *FVM_RESTRICT bnd, unsigned char *FVM_RESTRICT bnb) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  unsigned char b = 0;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int2 fj = lfj[q];
    if (bnd[fj.y >= 0 ? fj.y : ~fj.y] != NO_BOUNDARY) b = 1;
  }
  bnb[c] = b;
}

__global__ void k_link_tables(int n, const int *FVM_RESTRICT off, const int *FVM_RESTRICT lnk,
                              const int2 *FVM_RESTRICT s12, int2 *FVM_RESTRICT lfj) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int f = lnk[q];
    const int2 e = s12[f];
    lfj[q] = make_int2(f, e.x == c ? e.y : ~e.x);
  }
}

__global__ void k_shared_sync(int n, Params P, const Sched *FVM_RESTRICT S, const unsigned char *FVM_RESTRICT act,
                              const int *FVM_RESTRICT iscal, int *FVM_RESTRICT rung, double *FVM_RESTRICT tend) {
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
  S->inc[0] = 0;
  S->inc[1] = 0;
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
__device__ __forceinline__ void maxrung_dev(int n, const int *FVM_RESTRICT rung, int *FVM_RESTRICT out, int gt0_, int gnt_) {
  int r = 0;
  for (int i = gt0_; i < n; i += gnt_) r = max(r, rung[i]);
  for (int o = 16; o > 0; o >>= 1) r = max(r, __shfl_xor_sync(0xffffffffu, r, o));
  __shared__ int wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = max(r, wm[w]);
    atomicMax(out, r);
  }
}
__global__ void k_maxrung(int n, const int *FVM_RESTRICT rung, int *FVM_RESTRICT out) {
  maxrung_dev(n, rung, out, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// (V / (4 pi / 3))^(1/3) per cell, for Params::hcell.
__global__ void k_cell_radius(int n, const double *FVM_RESTRICT cvol, double *FVM_RESTRICT hcell) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) hcell[i] = pow(cvol[i] / (4.0 * M_PI / 3.0), 1.0 / 3.0);
}

// ---- init: compute_pvel + compute_timesteps(true) -------------------------
__global__ void k_init_dt(int n, Params P, const int *FVM_RESTRICT bnd, const double *FVM_RESTRICT U,
                          const double *FVM_RESTRICT volp, const double *FVM_RESTRICT vel,
                          const double *FVM_RESTRICT pos, double *FVM_RESTRICT dmin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double vmin = FVM_HUGE;
  if (i < n && !(P.halo && P.halo[i]))
    vmin = smin(extra_timestep(P, i, bnd, pos, vel),
                cell_timestep(P, i, false, nullptr, nullptr, bnd, U, volp, vel));
  for (int o = 16; o > 0; o >>= 1) vmin = smin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0) atomic_min_pos(dmin, vmin);
}

template <typename R>
__global__ void k_init_state(int n, const double *FVM_RESTRICT W, const double *FVM_RESTRICT cvol,
                             double *FVM_RESTRICT U, double *FVM_RESTRICT dU, R *FVM_RESTRICT Wrec,
                             double *FVM_RESTRICT volp) {
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
__global__ void k_limited_wrec(int n, const unsigned char *FVM_RESTRICT act, const R *FVM_RESTRICT Wrec,
                               const R *FVM_RESTRICT tau, double *FVM_RESTRICT out) {
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
__global__ void k_convert(long long n, const A *FVM_RESTRICT in, B *FVM_RESTRICT out) {
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
