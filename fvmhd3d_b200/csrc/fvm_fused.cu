// The persistent rung kernel: one cooperative launch runs a partial step (the
// cells of the active rungs and their neighbours, MPI/iterate.cpp:95-113 with
// MPI/Scheduler.h:108-154 choosing the rungs) from the slope limiter to the
// reconstruction, the stages separated by grid-wide barriers instead of
// kernel boundaries.  A step of the individual-timestep scheme that touches
// few cells is then one launch instead of some thirty dependent ones; the
// partial step's graph chooses between this kernel and the separate stage
// kernels on the device, by the step's involved-cell count.
//
// Every stage is the same device function the stage kernels call
// (fvm_device.cuh), over the same lists and in the same per-cell order, so
// both forms give the same bits.  This file includes fvm_device.cuh with
// FVM_RESTRICT empty: a stage here reads what earlier stages of the same
// launch wrote on other SMs, so nothing is promised read-only.
#define FVM_RESTRICT
#include "fvm_device.cuh"
#include "fvm_fused.h"

namespace {

// Lanes per cell in the cell passes of compute_update and compute_update0,
// the timestep and the adjust_timesteps marks: a small step has few cells,
// and each cell's walk over its ~16 faces is a chain of dependent loads;
// split over 8 lanes it is two loads deep.
constexpr int kCellGroup = 8;
// Lanes per cell and primitive pair in the slope limiter (five pairs per
// cell, so a cell takes 20 lanes).
constexpr int kLimGroup = 4;

// Polls of a grid barrier wait before it gives up (about 100 ns each): far
// above the longest stage of a step this kernel runs (the sequential
// adjust_timesteps sweep over at most its involved cells).
constexpr long long kBarrierPolls = 1ll << 24;

__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier over the nblocks working blocks of the launch (the
// first nblocks; the others have returned).  bar[0] counts arrivals
// (zero between barriers), bar[1] is the generation, which carries over from
// launch to launch: each block reads it on entry, and no barrier can complete
// before every block has arrived, so every block starts from the same value.
// Thread 0 of each block arrives after a release fence and waits, with
// bounded polls, for the generation its barrier completes; the last arrival
// resets the count and publishes the generation.  Returns false on every
// thread of the block if the wait gave up (err bit 1 set).
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned &gen, int *err, unsigned nblocks) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    const unsigned target = gen + 1;
    __threadfence();
    if (atomicAdd(&bar[0], 1u) == nblocks - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicExch(&bar[1], target);
    } else {
      long long it = 0;
      while (load_acquire(&bar[1]) != target) {
        if (++it > kBarrierPolls) {
          atomicOr(err, 1);
          ok = 0;
          break;
        }
        if (it > 4096) __nanosleep(64);  // short waits spin; long ones back off
      }
    }
    __threadfence();
  }
  gen++;
  return __syncthreads_and(ok) != 0;
}

__device__ __forceinline__ int vload(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

// The ascending list of the step's active non-boundary sites (site flag set
// by the mark stage), compacted from the ascending involved-cell list by one
// block: the order the sequential adjust_timesteps sweep visits them in.
__device__ void compact_sites(const int *clist, int ninv, const unsigned char *site, int *alist) {
  __shared__ int wsum[32];
  __shared__ int base;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < ninv; c0 += blockDim.x) {
    const int t = c0 + threadIdx.x;
    const int i = t < ninv ? clist[t] : -1;
    const bool f = i >= 0 && site[i] != 0;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[w] = __popc(b);
    __syncthreads();
    int o = base;
    for (int k = 0; k < w; k++) o += wsum[k];
    if (f) alist[o + __popc(b & ((1u << lane) - 1u))] = i;
    __syncthreads();
    if (threadIdx.x == 0)
      for (int k = 0; k < nw; k++) base += wsum[k];
    __syncthreads();
  }
}

// One partial step, limiter to reconstruction (the stage kernels' order in
// enq_limiter .. enq_recon), exact flux.  The step's active-face and
// involved-cell lists are built before the launch; never every cell is
// involved (such steps take the stage kernels).
template <typename R>
__global__ void __launch_bounds__(128, FVM_FLUX_MINB(R)) k_rung_step(FusedStep a) {
  const Params &P = a.P;
  const Dev &d = a.d;
  Sched *S = d.S;
  const int n = a.n, nf = a.nf;
  // Every block works: the stages of a small step are bound by the latency
  // of each thread's walk over its cell's faces, so more threads beat
  // cheaper barriers (one block per 64 involved cells measured 0.20 ms per
  // 200-cell step against 0.15 ms with the whole grid).
  const unsigned nwork = gridDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = (int)nwork * blockDim.x;
  // lane groups of the cell passes that split a cell's faces (same sums, in
  // the same order, as one thread per cell)
  const int gl = threadIdx.x & (kCellGroup - 1);
  const unsigned gmask = ((1u << kCellGroup) - 1u) << ((threadIdx.x & 31) & ~(kCellGroup - 1));
  unsigned gen = load_acquire(&a.gbar[1]);
#define FVM_GRID_SYNC() \
  if (!grid_barrier(a.gbar, gen, a.gerr, nwork)) return
  // the work arrays of adjust_timesteps start cleared for the step's
  // involved cells (the separate-kernel step clears them for every cell).
  // Every entry this step writes or reads is an involved cell's: marks and
  // work lists go to active cells and their neighbours, and the replays
  // below walk the involved cells only.
  {
    const int ninv = S->ninv;
    for (int t = gt; t < ninv; t += gn) {
      const int i = d.clist[t];
      d.hash[i] = 0;
      d.act0[i] = 0;
      d.awork[i] = 0;
      d.awork[(size_t)n + i] = 0;
    }
  }
  if (gt < 4) S->iscal[4 + gt] = 0;
  if (gt < 8) d.aflag[gt] = 0;
  // slope limiter over the involved cells
  {  // kLimGroup lanes per cell and primitive pair (a step with few cells,
     // never every cell active: the limiter's first pass always runs)
    constexpr int KH = CellTune<R>::KH_LIM, TPC = 10 / KH;
    const double t_global = S->t_global;
    const int units = TPC * S->ninv, gl4 = threadIdx.x & (kLimGroup - 1);
    const unsigned gmask4 = ((1u << kLimGroup) - 1u) << ((threadIdx.x & 31) & ~(kLimGroup - 1));
    for (int t = gt / kLimGroup; t < units; t += gn / kLimGroup)
      limiter_group<R, KH, kLimGroup>(d.clist[t / TPC], (t % TPC) * KH, gl4, gmask4, t_global, d.off, d.lfj,
                                      d.fflag, d.act, d.tlast, (const R *)d.Wrec, (R *)d.tau, (R *)d.fst,
                                      (const R *)d.lld);
  }
  FVM_GRID_SYNC();
  // compute_update: face fluxes over the active faces, then the cells
  corr_flux_dev<R, LM_EXACT>(nf, P, S, d.s12, d.geo, d.dr1, d.fflag, d.bnd, d.vel, d.tlast, (const R *)d.Wrec,
                             (const R *)d.fst, (R *)d.fcon, d.fcode, a.lb, d.flist, 1, gt, gn);
  FVM_GRID_SYNC();
  {  // the cells: kCellGroup lanes per cell, the walk over its faces split among them
    const double t_global = S->t_global;
    const int ninv = S->ninv;
    for (int t = gt / kCellGroup; t < ninv; t += gn / kCellGroup) {
      const int c = d.clist[t];
      corr_cell_group<R, kCellGroup>(c, gl, gmask, t_global, P, d.off, d.lfj, d.cvol, d.act, d.bnd, d.pos, d.tlast,
                                     d.volp, (const R *)d.Wrec, (const R *)d.tau, (const R *)d.fcon, d.fcode, d.U,
                                     d.dU, d.stepdU, d.counters, d.divb);
      // compute_pvel of the same cell (its own updated state; no stage
      // before the timestep reads a velocity)
      if (gl == 0) pvel_body(c, P, d.act, d.bnd, d.U, d.volp, d.cvol, d.ccen, d.pos, d.vel);
    }
  }
  FVM_GRID_SYNC();
  // compute_timesteps(false): CFL timestep and its minimum, halving,
  // adjust_timesteps (marks, parallel replays, sequential fallback), rungs
  timestep_group<kCellGroup>(P, d.off, d.lfj, d.act, d.bnd, d.U, d.volp, d.vel, d.pos, d.tlast, d.tend, d.dtl,
                             &S->dtmin, d.clist, S->ninv, gl, gmask, gt / kCellGroup, gn / kCellGroup);
  FVM_GRID_SYNC();
  halve_dev(n, d.act, &S->dtmin, d.dtl, d.clist, &S->ninv, gt, gn);
  FVM_GRID_SYNC();
  adjust_mark_group<kCellGroup>(d.off, d.lfj, d.act, d.bnd, d.dtl, d.hash, &S->iscal[4], d.act0, d.awork, d.clist,
                                S->ninv, gl, gmask, gt / kCellGroup, gn / kCellGroup);
  {  // active non-boundary sites (the count the separate-kernel step takes from its compaction)
    const int ninv = S->ninv;
    int cnt = 0;
    for (int t = gt; t < ninv; t += gn) cnt += d.act0[d.clist[t]] != 0;  // sites this thread marked
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&S->iscal[5], cnt);
  }
  FVM_GRID_SYNC();
  adjust_init_dev<kCellGroup>(n, d.off, d.lfj, d.act, &S->iscal[4], d.dtl, d.dt0, d.rdv, d.wrv, d.aflag, d.clist,
                              &S->ninv, gt, gn);
  FVM_GRID_SYNC();
  bool settled = false;
  for (int k = 0; k < ADJ_ITERS; k++) {
    adjust_replay_dev(n, k, d.off, d.lfj, d.lsort, d.lpart, d.act, d.dt0, d.rdv, d.wrv, d.dtl, d.aflag, d.awork, 0, gt,
                      gn, d.clist, S->ninv);
    FVM_GRID_SYNC();
    // stop once replay k changed nothing (settled) or every replay has run
    settled = vload(&d.aflag[k % 3]) == 0;
    if (settled || k + 1 >= ADJ_ITERS) break;
  }
  // adjust_restore_dev's decision, taken by every block from the same flags:
  // the sequential sweep runs from the initial timesteps when the replays did
  // not settle; otherwise the replays' timesteps stand and no barrier is
  // needed before the rungs
  {
    const bool fallback = !settled && vload(&d.aflag[(ADJ_ITERS - 1) % 3]) != 0;
    if (gt == 0) {
      if (settled) d.aflag[5] = 1;
      S->iscal[6] = vload(&d.aflag[3]);
      S->iscal[7] = fallback ? 1 : 0;
      if (fallback) d.aflag[4] = 1;
    }
    if (fallback) {
      const int ninv = S->ninv;
      for (int t = gt; t < ninv; t += gn) {
        const int u = d.clist[t];
        if (d.act[u] & (A_ACTIVE | A_LNGB)) d.dtl[u] = d.dt0[u];
      }
      FVM_GRID_SYNC();
      if (blockIdx.x == 0) {  // not settled: the sequential sweep
        compact_sites(d.clist, S->ninv, d.act0, d.alist);
        __syncthreads();
        if (threadIdx.x == 0) adjust_seq_dev(d.off, d.lnk, d.s12, d.alist, &S->iscal[5], &d.aflag[4], d.dtl);
      }
      FVM_GRID_SYNC();
    }
  }
  {  // rungs (and correct()) and distribute_fluid_update_data: both per cell, own data only
    const double t_global = S->t_global;
    const int min_rung = S->min_rung, ninv = S->ninv;
    for (int t = gt; t < ninv; t += gn) {
      const int i = d.clist[t];
      rungs_body<R>(i, t_global, min_rung, P, 0, d.act, d.hash, d.dtl, &S->dtmin, d.rung, d.tlast, d.tend,
                    (R *)d.Wrec, S->iscal, d.vel, d.opos, d.ovel);
      wst_body<R>(i, d.act, d.U, d.volp, (R *)d.Wst);
    }
  }
  FVM_GRID_SYNC();
  pred_flux_dev<R, LM_EXACT>(nf, P, d.s12, d.geo, d.dr1, d.fflag, d.bnd, d.vel, (const R *)d.Wst, (R *)d.fcon2,
                             d.fcode2, S, d.rung, a.lb, d.flist, 1, gt, gn);
  FVM_GRID_SYNC();
  {
    const double t_global = S->t_global;
    const int min_rung = S->min_rung, ninv = S->ninv;
    for (int t = gt / kCellGroup; t < ninv; t += gn / kCellGroup)
      pred_cell_group<R, kCellGroup>(d.clist[t], gl, gmask, t_global, min_rung, P, d.off, d.lfj, d.cvol, d.act,
                                     d.bnd, d.pos, d.U, (const R *)d.fcon2, d.fcode2, d.rung, d.tend,
                                     (R *)d.Wrec);
  }
  FVM_GRID_SYNC();
  recon_dev<R, CellTune<R>::KH_REC, CellTune<R>::MINB_REC>(n, P, S, d.off, d.lfj, d.cvol, d.act, d.bnd,
                                                           (const R *)d.Wst, d.rung, (R *)d.Wrec, d.perm,
                                                           (R *)d.mnmx, d.mz, (const R *)d.lrw, (const R *)d.lrd,
                                                           d.clist, d.bnb, gt, gn);
  if (gt == 0) S->fused_steps += 1;
#undef FVM_GRID_SYNC
}

template <typename R>
int blocks_per_sm() {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rung_step<R>, 128, 0) != cudaSuccess) return 0;
  return per;
}

}  // namespace

namespace fvm {

int fused_step_blocks_per_sm(bool fp32) { return fp32 ? blocks_per_sm<float>() : blocks_per_sm<double>(); }

cudaError_t fused_step_enqueue(const FusedStep &a, bool fp32, int grid, cudaStream_t st) {
  // The grid is the kernel's occupancy limit times the SM count and the
  // launch is the only work on its stream, so every block is resident at
  // once and the grid barriers can complete; were some not resident, the
  // bounded barriers would end the launch with err bit 1, not hang.
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  if (fp32)
    k_rung_step<float><<<grid, 128, 0, st>>>(a);
  else
    k_rung_step<double><<<grid, 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace fvm
