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
#include <climits>
#include <cstdlib>
#include <vector>
#include <string>
#include <algorithm>

using namespace fvm;

#include "fvm_device.cuh"
#include "fvm_fused.h"

// ============================== host context ================================

enum KernelId { KT_FLAGS = 0, KT_LIMITER, KT_CORR_FLUX, KT_CORR_CELL, KT_PVEL, KT_TIMESTEP, KT_RUNGS,
                KT_WST, KT_PRED_FLUX, KT_PRED_CELL, KT_RECON, KT_SYNC, KT_FUSED, KT_COUNT };
static const char *kKernelNames[KT_COUNT] = {"flags", "limiter", "corr_flux", "corr_cell", "pvel", "timestep",
                                             "rungs", "wst", "pred_flux", "pred_cell", "recon", "sync", "fused"};

// ---- mesh installation on the device (fvm_set_mesh) -----------------------
// The mesh contract is checked where the arrays land: err[k] receives the
// smallest index of a violation of kind k (INT_MAX when none), and the host
// reports the first kind found, in the order of MESH_ERR_*.
enum { MESH_ERR_CELL = 0, MESH_ERR_OFF, MESH_ERR_ID, MESH_ERR_SIDE, MESH_ERR_MISSING, MESH_ERR_COUNT };

// Per face: the cells in range and distinct; (s1, s2), unit normal and area,
// centroid.  The area is the rounded sqrt of the rounded sum of squares with
// no contraction, as the host computes it.
__global__ void k_mesh_faces(int nf, int ncell, const int *__restrict__ s1, const int *__restrict__ s2,
                             const double *__restrict__ n3, const double *__restrict__ c3, int2 *__restrict__ s12,
                             double4 *__restrict__ geo, double4 *__restrict__ cen, int *__restrict__ err) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int a = s1[f], b = s2[f];
  if (a < 0 || a >= ncell || b < 0 || b >= ncell || a == b) atomicMin(&err[MESH_ERR_CELL], f);
  s12[f] = make_int2(a, b);
  const double v0 = n3[3 * (size_t)f], v1 = n3[3 * (size_t)f + 1], v2 = n3[3 * (size_t)f + 2];
  const double area = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2)));
  const double ia = 1.0 / area;
  geo[f] = make_double4(v0 * ia, v1 * ia, v2 * ia, area);
  cen[f] = make_double4(c3[3 * (size_t)f], c3[3 * (size_t)f + 1], c3[3 * (size_t)f + 2], 0.0);
}

// Per cell: CSR offsets within [0, nl] and not decreasing; as int.
__global__ void k_mesh_offsets(int ncell, long long nl, const long long *__restrict__ off64, int *__restrict__ off,
                               int *__restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > ncell) return;
  const long long o = off64[i];
  if (o < 0 || o > nl || (i < ncell && off64[i + 1] < o)) atomicMin(&err[MESH_ERR_OFF], i);
  off[i] = (int)(o < 0 ? 0 : (o > nl ? nl : o));
}

// Per cell (offsets checked): its face ids in range, each face listed by its
// own two cells only, once each (flink[2 f + side] = the link, -1 before).
__global__ void k_mesh_links(int ncell, int nf, const int *__restrict__ off, const int *__restrict__ ids,
                             const int2 *__restrict__ s12, int *__restrict__ lnk, int *__restrict__ flink,
                             int *__restrict__ err) {
  const int c0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (c0 >= ncell) return;
  for (int q = off[c0]; q < off[c0 + 1]; q++) {
    const int f = ids[q];
    lnk[q] = f;
    if (f < 0 || f >= nf) { atomicMin(&err[MESH_ERR_ID], q); continue; }
    const int2 e = s12[f];
    const int side = e.x == c0 ? 0 : (e.y == c0 ? 1 : -1);
    if (side < 0 || atomicCAS(&flink[2 * (size_t)f + side], -1, q) != -1) atomicMin(&err[MESH_ERR_SIDE], f);
  }
}

// Per face: both sides listed; each link's partner link.
__global__ void k_mesh_partners(int nf, const int *__restrict__ flink, int *__restrict__ lpart, int *__restrict__ err) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int a = flink[2 * (size_t)f], b = flink[2 * (size_t)f + 1];
  if (a < 0 || b < 0) { atomicMin(&err[MESH_ERR_MISSING], f); return; }
  lpart[a] = b;
  lpart[b] = a;
}

// Per cell: its links ordered by ascending neighbour index (insertion sort,
// stable; a cell has a few tens of faces), and the identity thread-to-cell map.
__global__ void k_mesh_sort(int ncell, const int *__restrict__ off, const int *__restrict__ lnk,
                            const int2 *__restrict__ s12, int *__restrict__ lsort, int *__restrict__ perm) {
  const int c0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (c0 >= ncell) return;
  perm[c0] = c0;
  const int q0 = off[c0], q1 = off[c0 + 1];
  auto nb = [&](int q) {
    const int2 e = s12[lnk[q]];
    return e.x == c0 ? e.y : e.x;
  };
  for (int q = q0; q < q1; q++) {
    const int key = nb(q);
    int p = q;
    while (p > q0 && nb(lsort[p - 1]) > key) {
      lsort[p] = lsort[p - 1];
      p--;
    }
    lsort[p] = q;
  }
}

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
  long long cap_n = 0, cap_f = 0, cap_l = 0;  // room of the mesh arrays (alloc_mesh)
  // scheduler (MPI/Scheduler.h)
  unsigned long long tsysU;
  int min_rung, max_rung;
  double t_global;
  bool have_mesh, have_state, in_step;
  bool have_geom = false;  // generator positions and the tables built from them belong to the mesh
  bool fp32;    // bulk (reconstruction, limiter, flux) in single precision
  size_t rb;    // bytes of one bulk value
  unsigned long long cur_flags;
  Dev d;
  bool keep_step_dU;
  float last_ms;
  // one captured step per mode (shared / individual), replayed by fvm_run
  cudaGraphExec_t graph[2];
  Sched hS;  // host copy of the device scheduler, refreshed after synchronisation
  // learned flux network: image of the FP16 weights and bias operands
  unsigned char *mlp_img = nullptr;
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
  // persistent rung kernel (fvm_fused.cu): captured partial steps whose
  // involved cells number at most fused_max run as one launch (0: never)
  int fused_max = 0;
  // partial steps whose active cells and their links number at most inc_max
  // build their lists incrementally (0: always the pass over every face;
  // -1: automatic, see inc_limit)
  int inc_max = -1;
  int fused_bpsm = 0;          // its resident blocks per SM (queried outside capture)
  // the reduction of the timestep minimum over ranks (fvm_set_reduce)
  fvm_reduce_fn reduce = nullptr;
  void *reduce_user = nullptr;
  cudaStream_t aux = nullptr;  // captures the branches of the fused/stage choice
  // fvm_step_host: the copy stream and the events that order its copies
  // against the stage kernels (created on first use)
  cudaStream_t cpy = nullptr;
  cudaEvent_t hev[5] = {};
  unsigned *gbar = nullptr;    // its grid barrier
  int *gerr = nullptr;         // its error bits
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
  if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->gbar, 2 * sizeof(unsigned)) != cudaSuccess || cudaMalloc(&c->gerr, sizeof(int)) != cudaSuccess ||
      cudaMemset(c->gerr, 0, sizeof(int)) != cudaSuccess || cudaMemset(c->gbar, 0, 2 * sizeof(unsigned)) != cudaSuccess) {
    fvm_destroy(c);
    return nullptr;
  }
  c->fused_bpsm = fused_step_blocks_per_sm(c->fp32);
  return c;
}

void fvm_destroy(fvm_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  drop_graphs(c);
  free_all(c);
  if (c->mlp_img) cudaFree(c->mlp_img);
  if (c->mlp_err) cudaFree(c->mlp_err);
  if (c->mlp_param) cudaFree(c->mlp_param);
  for (int k = 0; k < 2 * KT_COUNT; k++) cudaEventDestroy(c->kev[k]);
  if (c->gbar) cudaFree(c->gbar);
  if (c->gerr) cudaFree(c->gerr);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  if (c->aux) cudaStreamDestroy(c->aux);
  if (c->cpy) cudaStreamDestroy(c->cpy);
  for (cudaEvent_t e : c->hev)
    if (e) cudaEventDestroy(e);
  cudaStreamDestroy(c->st);
  delete c;
}

const char *fvm_last_error(const fvm_ctx *c) { return c ? c->err.c_str() : "null context"; }

// Device arrays of a mesh with room for ncell cells, nface faces and nl
// links (cap_* record the room; a mesh that fits reuses them).
static int alloc_mesh(fvm_ctx *c, long long ncell, long long nface, long long nl) {
  free_all(c);
  c->cap_n = c->cap_f = c->cap_l = 0;
  int rc = 0;
  Dev &d = c->d;
  rc |= dalloc(c, &d.s12, nface); rc |= dalloc(c, &d.geo, nface); rc |= dalloc(c, &d.cen, nface);
  rc |= dalloc(c, &d.dr1, nface); rc |= dalloc(c, &d.dr2, nface); rc |= dalloc(c, &d.fflag, nface);
  rc |= dalloc_bytes(c, &d.fst, 20 * c->rb * (size_t)nface);
  rc |= dalloc(c, &d.cvol, ncell); rc |= dalloc(c, &d.ccen, 3 * (size_t)ncell);
  rc |= dalloc(c, &d.hcell, ncell); rc |= dalloc(c, &d.halo, ncell);
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
  rc |= dalloc(c, &d.ilist, ncell);
  const long long ibits_words = (ncell + 31) / 32;
  rc |= dalloc(c, &d.ibits, ibits_words);
  rc |= dalloc(c, &d.icount, std::max(INC_BLOCKS, SITE_BLOCKS));
  rc |= dalloc(c, &d.bnb, ncell);
  rc |= dalloc_bytes(c, &d.tau, 10 * c->rb * (size_t)ncell);
  rc |= dalloc_bytes(c, &d.fcon, 14 * c->rb * (size_t)nface);
  rc |= dalloc_bytes(c, &d.fcon2, 14 * c->rb * (size_t)nface);
  rc |= dalloc_bytes(c, &d.Wst, 10 * c->rb * (size_t)ncell);
  rc |= dalloc(c, &d.dtl, ncell);
  if (c->keep_step_dU) rc |= dalloc(c, &d.stepdU, 14 * (size_t)ncell);
  rc |= dalloc(c, &d.S, 1); rc |= dalloc(c, &d.counters, 4);
  if (rc) { free_all(c); return FVM_ENOMEM; }
  // zero between steps (ibits), and cleared per step only where a step
  // works (the adjust_timesteps work arrays of partial steps)
  if (cudaMemset(d.ibits, 0, sizeof(unsigned) * ibits_words) != cudaSuccess ||
      cudaMemset(d.hash, 0, ncell) != cudaSuccess || cudaMemset(d.act0, 0, ncell) != cudaSuccess ||
      cudaMemset(d.awork, 0, 2 * ncell) != cudaSuccess) {
    free_all(c);
    return FVM_ENOMEM;
  }
  c->cap_n = ncell;
  c->cap_f = nface;
  c->cap_l = nl;
  c->P.hcell = d.hcell;
  return 0;
}

// Releases the learned-flux buffers (sized by the face count of the mesh
// they were made for).
static void free_learn_buffers(fvm_ctx *c) {
  Dev &d = c->d;
  void **bufs[] = {&d.lX, &d.lY, &d.lface, &d.lcount, &d.lstats, &d.lhx, &d.lhy, &d.lhcount, &d.lnorm};
  for (void **b : bufs) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
}

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
  if ((ncell + CB - 1) / CB > CB * 16) { c->err = "fvm_set_mesh: more than 16M cells"; return FVM_ERANGE; }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);
  c->have_mesh = false;
  c->have_state = false;
  c->have_geom = false;
  c->P.halo = nullptr;
  c->learn_mode = 0;
  c->lb = LearnBuf{};
  free_learn_buffers(c);
  // a mesh that fits the arrays of the last one reuses them (a host that
  // rebuilds its mesh every step installs one of about the same size);
  // otherwise they are made anew with a little room to grow
  if (ncell > c->cap_n || nface > c->cap_f || nl > c->cap_l) {
    const int rc = alloc_mesh(c, ncell + ncell / 32 + 64, nface + nface / 32 + 256, nl + nl / 32 + 512);
    if (rc) return rc;
  }
  c->n = ncell;
  c->nf = nface;
  c->nl = nl;
  Dev &d = c->d;
  // the host arrays, staged as they are; the device lays them out and checks
  // them (mesh kernels above)
  const size_t b_s = sizeof(int) * (size_t)nface, b_v = sizeof(double) * 3 * (size_t)nface,
               b_o = sizeof(long long) * ((size_t)ncell + 1), b_i = sizeof(int) * (size_t)nl,
               b_fl = 2 * sizeof(int) * (size_t)nface, b_e = 64;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  char *stage = nullptr;
  CK(cudaMallocAsync((void **)&stage, 2 * up(b_s) + 2 * up(b_v) + up(b_o) + up(b_i) + up(b_fl) + b_e, c->st));
  int *ds1 = (int *)stage, *ds2 = (int *)(stage + up(b_s));
  double *dn = (double *)(stage + 2 * up(b_s)), *dc = (double *)(stage + 2 * up(b_s) + up(b_v));
  long long *doff = (long long *)(stage + 2 * up(b_s) + 2 * up(b_v));
  int *dids = (int *)((char *)doff + up(b_o));
  int *flink = (int *)((char *)dids + up(b_i));
  int *derr = (int *)((char *)flink + up(b_fl));
  int herr[MESH_ERR_COUNT];
  auto finish = [&](int rc) {
    cudaFreeAsync(stage, c->st);
    const cudaError_t e = cudaStreamSynchronize(c->st);
    if (rc == 0 && e != cudaSuccess) {
      c->err = std::string("fvm_set_mesh: ") + cudaGetErrorString(e);
      return (int)FVM_ECUDA;
    }
    return rc;
  };
  auto fetch_errors = [&]() -> int {
    if (cudaMemcpyAsync(herr, derr, sizeof(herr), cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
      c->err = "fvm_set_mesh: reading the mesh checks failed";
      return FVM_ECUDA;
    }
    const char *what[MESH_ERR_COUNT] = {"face %d has a bad cell index", "CSR offsets of cell %d out of order or range",
                                        "bad face id at link %d of the cell lists",
                                        "face %d listed by a cell that is not its side, or twice",
                                        "face %d missing from a cell's face list"};
    for (int k = 0; k < MESH_ERR_COUNT; k++)
      if (herr[k] != 0x7f7f7f7f) {
        char buf[160];
        snprintf(buf, sizeof(buf), what[k], herr[k]);
        c->err = std::string("fvm_set_mesh: ") + buf;
        return FVM_EINVAL;
      }
    return 0;
  };
  CK(cudaMemcpyAsync(ds1, s1, b_s, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(ds2, s2, b_s, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dn, n, b_v, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dc, centroid, b_v, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(doff, off, b_o, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dids, ids, b_i, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d.cvol, cell_volume, sizeof(double) * ncell, cudaMemcpyHostToDevice, c->st));
  k_cell_radius<<<nblk(ncell, 256), 256, 0, c->st>>>(ncell, d.cvol, d.hcell);
  LAUNCH_CHECK();
  CK(cudaMemcpyAsync(d.ccen, cell_centroid, sizeof(double) * 3 * ncell, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(derr, 0x7f, sizeof(herr), c->st));
  CK(cudaMemsetAsync(flink, 0xff, b_fl, c->st));
  if (nface > 0)
    k_mesh_faces<<<nblk(nface, 256), 256, 0, c->st>>>(nface, ncell, ds1, ds2, dn, dc, d.s12, d.geo, d.cen, derr);
  k_mesh_offsets<<<nblk(ncell + 1, 256), 256, 0, c->st>>>(ncell, nl, doff, d.off, derr);
  LAUNCH_CHECK();
  int rc = fetch_errors();
  if (rc) return finish(rc);
  k_mesh_links<<<nblk(ncell, 128), 128, 0, c->st>>>(ncell, nface, d.off, dids, d.s12, d.lnk, flink, derr);
  if (nface > 0) k_mesh_partners<<<nblk(nface, 256), 256, 0, c->st>>>(nface, flink, d.lpart, derr);
  LAUNCH_CHECK();
  if ((rc = fetch_errors())) return finish(rc);
  k_mesh_sort<<<nblk(ncell, 128), 128, 0, c->st>>>(ncell, d.off, d.lnk, d.s12, d.lsort, d.perm);
  k_link_tables<<<nblk(ncell, 256), 256, 0, c->st>>>(ncell, d.off, d.lnk, d.s12, d.lfj);
  LAUNCH_CHECK();
  // no face active yet, every face coded F_OFF (k_faceflags keeps this so for
  // the faces it turns inactive)
  CK(cudaMemsetAsync(d.fflag, 0, nface, c->st));
  CK(cudaMemsetAsync(d.fcode, F_OFF, nface, c->st));
  CK(cudaMemsetAsync(d.fcode2, F_OFF, nface, c->st));
  CK(cudaMemsetAsync(d.counters, 0, 4 * sizeof(unsigned long long), c->st));
  if ((rc = finish(0))) return rc;
  c->have_mesh = true;
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

// Generator positions and boundary codes of the installed mesh, and what is
// built from them: the boundary-neighbour flags, the face offsets and the
// per-link tables of the limiter and the reconstruction.
static int enq_positions(fvm_ctx *c, const double *pos, const int *bnd) {
  const int n = c->n;
  Dev &d = c->d;
  CK(cudaMemcpyAsync(d.pos, pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, c->st));
  if (bnd) CK(cudaMemcpyAsync(d.bnd, bnd, sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
  else CK(cudaMemsetAsync(d.bnd, 0, sizeof(int) * n, c->st));
  k_bnd_neighbours<<<nblk(n, 256), 256, 0, c->st>>>(n, d.off, d.lfj, d.bnd, d.bnb);
  LAUNCH_CHECK();
  k_face_geom<<<nblk(c->nf, 256), 256, 0, c->st>>>(c->nf, c->P, d.s12, d.geo, d.cen, d.pos, d.dr1, d.dr2);
  LAUNCH_CHECK();
  BULK(k_link_recon<R><<<nblk(n, 256), 256, 0, c->st>>>(n, c->P, d.off, d.lfj, d.geo, d.dr1, d.dr2, (R *)d.lrw,
                                                        (R *)d.lrd, (R *)d.lld));
  LAUNCH_CHECK();
  c->have_geom = true;
  return 0;
}

int fvm_set_positions(fvm_ctx *c, const double *pos, const int *bnd) {
  if (!c || !pos) { if (c) c->err = "fvm_set_positions: bad argument"; return FVM_EINVAL; }
  if (!c->have_mesh) { c->err = "fvm_set_positions: no mesh"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_set_positions: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const int rc = enq_positions(c, pos, bnd);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->st));
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
  int rc = enq_positions(c, pos, bnd);
  if (rc) { cudaFree(dW); return rc; }
  CK(cudaMemsetAsync(d.vel, 0, sizeof(double) * 3 * (size_t)n, c->st));
  CK(cudaMemsetAsync(d.tlast, 0, sizeof(double) * n, c->st));

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
  if (c->reduce && c->reduce(c->reduce_user, &dtmin) != 0) {
    c->err = "fvm_init_problem: the timestep reduction failed";
    return FVM_EINVAL;
  }
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
  if (!c->have_geom) { c->err = "fvm_set_state: no generator positions for this mesh (fvm_set_positions)"; return FVM_ENOMESH; }
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

// The flags and lists of a partial step by a pass over every face and cell.
static int enq_lists_meshwide(fvm_ctx *c) {
  Dev &d = c->d;
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
  return 0;
}

// The same flags and lists built from the active cells' links (k_inc_*).
static int enq_lists_incremental(fvm_ctx *c) {
  Dev &d = c->d;
  // a warp per cell, 8 per 256-thread block, on a fixed grid (the cell
  // counts are known only on the device)
  const int grid = 8 * c->sms;
  k_inc_mark<<<grid, 256, 0, c->st>>>(d.off, d.lfj, d.act, d.S, d.ilist, d.ibits);
  LAUNCH_CHECK();
  k_inc_count<<<INC_BLOCKS, 256, 0, c->st>>>(c->n, d.ibits, d.icount);
  LAUNCH_CHECK();
  k_inc_cells<<<INC_BLOCKS, 256, 0, c->st>>>(c->n, d.S, d.ibits, d.icount, d.clist);
  LAUNCH_CHECK();
  k_inc_faces<<<grid, 256, 0, c->st>>>(d.off, d.lfj, d.s12, d.act, d.bnd, d.fflag, d.fcode, d.fcode2, d.S, d.clist,
                                       d.flist);
  LAUNCH_CHECK();
  return 0;
}

// The bound of incremental list building in cells plus links (0: off).
// Automatic: 1/256 of the mesh's cells plus links, at least 8192.  The
// incremental active-face list is in the order the faces were found, and on
// the 1M-cell disk steps of 65K active cells took 4% longer with it (the
// flux passes lose the face order's locality) while 200-cell steps gained
// 0.08 ms; the bound keeps it to the small steps.
static int inc_limit(const fvm_ctx *c) {
  if (c->inc_max >= 0) return c->inc_max;
  return (int)std::min<long long>(INT_MAX, std::max<long long>(8192, ((long long)c->n + c->nl) / 256));
}

// Sets the branch of a captured partial step's list building: incremental
// when the active cells and their links number at most inc_max.
__global__ void k_inc_choose(Sched *S, int inc_max, cudaGraphConditionalHandle h) {
  const int small = S->iscal[1] + S->inc[0] <= inc_max;
  S->inc[1] = small;
  S->inc_steps += small;
  cudaGraphSetConditional(h, small ? 1u : 0u);
}
__global__ void k_inc_set(Sched *S) {
  S->inc[1] = 1;
  S->inc_steps += 1;
}

// Captured partial step: an if/else graph node whose branches build the
// lists incrementally or by the pass over every face (same lists, same bits).
static int enq_lists_choice(fvm_ctx *c) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  k_inc_choose<<<1, 1, 0, c->st>>>(c->d.S, inc_limit(c), h);
  LAUNCH_CHECK();
  CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 2;
  cudaGraphNode_t cn;
  CK(cudaGraphAddNode(&cn, g, deps, nd, &cp));
  cudaGraph_t body_inc = cp.conditional.phGraph_out[0], body_mesh = cp.conditional.phGraph_out[1];
  // each branch is captured with the auxiliary stream standing in for the
  // context's
  int rc = 0;
  for (int b = 0; b < 2 && !rc; b++) {
    std::swap(c->st, c->aux);
    const cudaError_t be = cudaStreamBeginCaptureToGraph(c->st, b == 0 ? body_inc : body_mesh, nullptr, nullptr, 0,
                                                         cudaStreamCaptureModeRelaxed);
    cudaError_t ee = cudaSuccess;
    cudaGraph_t done = nullptr;
    if (be == cudaSuccess) {
      rc = b == 0 ? enq_lists_incremental(c) : enq_lists_meshwide(c);
      ee = cudaStreamEndCapture(c->st, &done);
    }
    std::swap(c->st, c->aux);
    CK(be);
    if (rc) return rc;
    CK(ee);
  }
  CK(cudaStreamUpdateCaptureDependencies(c->st, &cn, 1, cudaStreamSetCaptureDependencies));
  return 0;
}

static int enq_begin(fvm_ctx *c) {
  const int n = c->n;
  Dev &d = c->d;
  kt_begin(c, KT_FLAGS);
  k_sched_begin<<<1, 1, 0, c->st>>>(c->P, d.S);
  LAUNCH_CHECK();
  const bool inc = c->use_flist && inc_limit(c) > 0;
  k_active<<<nblk(n, 256), 256, 0, c->st>>>(n, d.rung, d.S, d.act, &d.S->iscal[1], d.off, inc ? d.ilist : nullptr,
                                            &d.S->inc[0]);
  LAUNCH_CHECK();
  int rc = 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->st, &cs));
  if (inc && cs == cudaStreamCaptureStatusActive && !c->prof) {
    rc = enq_lists_choice(c);
  } else if (inc && cs == cudaStreamCaptureStatusNone) {
    // an eager step makes the same choice on the host
    int cnt[2] = {0, 0};
    CK(cudaMemcpyAsync(&cnt[0], &d.S->iscal[1], sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&cnt[1], &d.S->inc[0], sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if ((long long)cnt[0] + cnt[1] <= inc_limit(c)) {
      k_inc_set<<<1, 1, 0, c->st>>>(d.S);
      LAUNCH_CHECK();
      rc = enq_lists_incremental(c);
    } else {
      rc = enq_lists_meshwide(c);
    }
  } else {
    rc = enq_lists_meshwide(c);
  }
  if (rc) return rc;
  kt_end(c, KT_FLAGS);
  return 0;
}

// The staged limiter, instantiation MINB (resident blocks per SM).  A partial
// step launches it on a grid of resident blocks (it returns at once unless
// every cell is active); a global step on one block per cell block.
extern "C++" {
template <typename R, int MINB>
static int limiter_st_launch(fvm_ctx *c) {
  Dev &d = c->d;
  constexpr int KH = CellTune<R>::KH_LIM;
  // the attribute is per device: set once for each device a context uses
  static bool attr[kMaxDevices] = {};
  if (c->device < 0 || c->device >= kMaxDevices) { c->err = "device index out of range"; return FVM_EINVAL; }
  if (!attr[c->device]) {
    CK(cudaFuncSetAttribute(k_limiter_st<R, KH, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            limiter_stage_bytes<R, KH>()));
    attr[c->device] = true;
  }
  const long long ncb = nblk(c->n, limiter_cst<KH>());
  const long long grid = c->use_flist ? std::min<long long>(ncb, (long long)MINB * c->sms) : ncb;
  k_limiter_st<R, KH, MINB><<<(unsigned)grid, 128, limiter_stage_bytes<R, KH>(), c->st>>>(
      c->n, c->P, d.S, d.off, d.lnk, d.lfj, d.s12, d.geo, d.dr1, d.fflag, d.act, d.tlast, (const R *)d.Wrec,
      (R *)d.tau, (R *)d.fst, d.perm, (const R *)d.mnmx, d.mz, c->use_flist, (const R *)d.lld);
  return 0;
}
}  // extern "C++"

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
      const int rc = c->use_flist ? limiter_st_launch<R, CellTune<R>::MINB_LIM>(c)
                                  : limiter_st_launch<R, CellTune<R>::MINB_LIM_G>(c);
      if (rc) return rc;
    }));
    LAUNCH_CHECK();
  }
  if (!staged || c->use_flist) {
    const int bs = c->tune.bs_cell2;
#define LIMITER_LIST(MB)                                                                                       \
  BULK(k_limiter<R, CellTune<R>::KH_LIM, MB>                                                                  \
       <<<sgrid(c, (long long)(10 / CellTune<R>::KH_LIM) * c->n, bs), bs, 0, c->st>>>(                         \
           c->n, c->P, d.S, d.off, d.lnk, d.lfj, d.s12, d.geo, d.dr1, d.fflag, d.act, d.tlast, (const R *)d.Wrec, \
           (R *)d.tau, (R *)d.fst, d.perm, (const R *)d.mnmx, d.mz, c->use_flist ? d.clist : nullptr,          \
           staged && c->use_flist, (const R *)d.lld))
    if (c->use_flist) LIMITER_LIST(CellTune<R>::MINB_LIM);
    else LIMITER_LIST(CellTune<R>::MINB_LIM_G);
#undef LIMITER_LIST
  }
  LAUNCH_CHECK();
  kt_end(c, KT_LIMITER);
  return 0;
}

static int mlp_launch_dev(fvm_ctx *c, int nmax, const int *n_dev, const __half *X, float *Y);

static int enq_corr_flux(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_CORR_FLUX);
  const LearnBuf &lb = c->lb;
#define CORR_FLUX(MODE, GRID, ...)                                                                              \
  BULK(k_corr_flux<R, MODE, ##__VA_ARGS__><<<GRID, c->tune.bs_face, 0, c->st>>>(c->nf, c->P, d.S, d.s12, d.geo, d.dr1, d.fflag, d.bnd, d.vel, \
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
  } else if (c->use_flist) {
    CORR_FLUX(LM_EXACT, sgrid(c, c->nf, c->tune.bs_face));
  } else {  // a global step: the instantiation with more resident blocks
    CORR_FLUX(LM_EXACT, sgrid(c, c->nf, c->tune.bs_face), FVM_GLOBAL_FLUX_MINB(R));
  }
#undef CORR_FLUX
  LAUNCH_CHECK();
  kt_end(c, KT_CORR_FLUX);
  return 0;
}

static int enq_corr_cell(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_CORR_CELL);
#define CORR_CELL(K)                                                                                           \
  BULK(K<R><<<sgrid(c, c->n, c->tune.bs_cell), c->tune.bs_cell, 0, c->st>>>(                                   \
      c->n, c->P, d.S, d.off, d.lfj, d.s12, d.cvol, d.act, d.bnd, d.pos, d.tlast, d.volp, (const R *)d.Wrec,     \
      (const R *)d.tau, (const R *)d.fcon, d.fcode, d.U, d.dU, d.stepdU, d.counters, d.perm, d.divb,            \
      c->use_flist ? d.clist : nullptr))
  if (c->use_flist || !c->fp32) CORR_CELL(k_corr_cell);
  else CORR_CELL(k_corr_cell_g);  // an FP32 global step: more resident blocks
#undef CORR_CELL
  LAUNCH_CHECK();
  kt_end(c, KT_CORR_CELL);
  return 0;
}

// compute_update: the face fluxes, then the cells.
static int enq_update(fvm_ctx *c) {
  const int rc = enq_corr_flux(c);
  return rc ? rc : enq_corr_cell(c);
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
  if (c->reduce) {  // the minimum over ranks (MPI/compute_timestep.cpp:101)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(c->st, &cs));
    if (cs != cudaStreamCaptureStatusNone) { c->err = "the timestep reduction needs eager steps"; return FVM_EINVAL; }
    double v = 0.0;
    CK(cudaMemcpyAsync(&v, &d.S->dtmin, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (c->reduce(c->reduce_user, &v) != 0) { c->err = "the timestep reduction failed"; return FVM_EINVAL; }
    CK(cudaMemcpyAsync(&d.S->dtmin, &v, sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (!shared) {
    k_halve<<<sgrid(c, n, 256), 256, 0, c->st>>>(n, d.act, &d.S->dtmin, d.dtl, cl, &d.S->ninv);
    LAUNCH_CHECK();
    CK(cudaMemsetAsync(&d.S->iscal[4], 0, 4 * sizeof(int), c->st));
    if (cl) {  // the work arrays and the site list over the involved cells only
      k_adjust_clear<<<sgrid(c, n, 256), 256, 0, c->st>>>(n, cl, &d.S->ninv, d.hash, d.act0, d.awork);
      LAUNCH_CHECK();
    } else {
      CK(cudaMemsetAsync(d.hash, 0, n, c->st));
      CK(cudaMemsetAsync(d.awork, 0, 2 * (size_t)n, c->st));
      CK(cudaMemsetAsync(d.act0, 0, n, c->st));
    }
    k_adjust_mark<<<sgrid(c, 8LL * n, 128), 128, 0, c->st>>>(n, d.off, d.lfj, d.act, d.bnd, d.dtl, d.hash,
                                                      &d.S->iscal[4], d.act0, d.awork, cl, &d.S->ninv);
    LAUNCH_CHECK();
    if (cl) {
      k_site_count<<<SITE_BLOCKS, 256, 0, c->st>>>(n, cl, &d.S->ninv, d.act0, d.icount);
      LAUNCH_CHECK();
      k_site_place<<<SITE_BLOCKS, 256, 0, c->st>>>(n, cl, &d.S->ninv, d.act0, d.icount, d.alist, &d.S->iscal[5]);
      LAUNCH_CHECK();
    } else {
      const int nb = (int)((n + CB - 1) / CB);
      k_count_flags<<<nb, CB, 0, c->st>>>(n, d.act0, d.bcount);
      LAUNCH_CHECK();
      k_scan_counts<<<1, CB, 0, c->st>>>(nb, d.bcount, &d.S->iscal[5]);
      LAUNCH_CHECK();
      k_place_flags<<<nb, CB, 0, c->st>>>(n, d.act0, d.bcount, d.alist);
      LAUNCH_CHECK();
    }
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
      const int *ulist = cl, *ucount = cl ? &d.S->ninv : nullptr;  // the replays walk the involved cells
      void *ra[] = {(void *)&n, &k0, &d.off, &d.lfj, &d.lsort, &d.lpart, &d.act, &d.dt0, &d.rdv, &d.wrv, &d.dtl,
                    &d.aflag, &d.awork, &kdev, &ulist, &ucount};
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
                                                  d.dtl, d.aflag, d.awork, 0, cl, cl ? &d.S->ninv : nullptr);
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
#define PRED_FLUX(MODE, GRID, ...)                                                                            \
  BULK(k_pred_flux<R, MODE, ##__VA_ARGS__><<<GRID, c->tune.bs_face, 0, c->st>>>(c->nf, c->P, d.s12, d.geo, d.dr1, d.fflag, d.bnd, \
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
  } else if (c->use_flist) {
    PRED_FLUX(LM_EXACT, sgrid(c, c->nf, c->tune.bs_face));
  } else {  // a global step: the instantiation with more resident blocks
    PRED_FLUX(LM_EXACT, sgrid(c, c->nf, c->tune.bs_face), FVM_GLOBAL_FLUX_MINB(R));
  }
#undef PRED_FLUX
  LAUNCH_CHECK();
  kt_end(c, KT_PRED_FLUX);
  return 0;
}

static int enq_recon(fvm_ctx *c) {
  Dev &d = c->d;
  kt_begin(c, KT_PRED_CELL);
#define PRED_CELL(K)                                                                                           \
  BULK(K<R><<<sgrid(c, c->n, c->tune.bs_cell), c->tune.bs_cell, 0, c->st>>>(                                   \
      c->n, c->P, d.S, d.off, d.lfj, d.s12, d.cvol, d.act, d.bnd, d.pos, d.U, (const R *)d.fcon2, d.fcode2,      \
      d.rung, d.tend, (R *)d.Wrec, d.perm, c->use_flist ? d.clist : nullptr))
  if (c->use_flist || !c->fp32) PRED_CELL(k_pred_cell);
  else PRED_CELL(k_pred_cell_g);  // an FP32 global step: more resident blocks
#undef PRED_CELL
  LAUNCH_CHECK();
  kt_end(c, KT_PRED_CELL);
  kt_begin(c, KT_RECON);
#define RECON(MB)                                                                                              \
  BULK(k_recon<R, CellTune<R>::KH_REC, MB>                                                                     \
       <<<sgrid(c, (long long)(10 / CellTune<R>::KH_REC) * c->n, c->tune.bs_cell2), c->tune.bs_cell2, 0, c->st>>>( \
           c->n, c->P, d.S, d.off, d.lfj, d.cvol, d.act, d.bnd, (const R *)d.Wst, d.rung, (R *)d.Wrec, d.perm,   \
           (R *)d.mnmx, d.mz, (const R *)d.lrw, (const R *)d.lrd, c->use_flist ? d.clist : nullptr, d.bnb))
  if (c->use_flist) RECON(CellTune<R>::MINB_REC);
  else RECON(CellTune<R>::MINB_REC_G);  // a global step: more resident blocks (FP32)
#undef RECON
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

// The step's stages from the slope limiter to the reconstruction, as
// separate kernels.
static int enq_stages(fvm_ctx *c, int shared) {
  int rc;
  if ((rc = enq_limiter(c))) return rc;
  if ((rc = enq_update(c))) return rc;
  if ((rc = enq_pvel(c))) return rc;
  if ((rc = enq_timesteps(c, shared))) return rc;
  if ((rc = enq_collect(c))) return rc;
  if ((rc = enq_update0(c))) return rc;
  return enq_recon(c);
}

// Blocks per SM of the persistent rung kernel's grid (at most its resident
// limit): a step it runs involves few cells, and fewer blocks make each grid
// barrier cheaper.
#ifndef FVM_FUSED_BPSM
#define FVM_FUSED_BPSM 1
#endif

// Sets the branch of a captured partial step: the persistent rung kernel
// when the step involves at most max_cells cells (and not every cell), else
// the stage kernels.
__global__ void k_fused_choose(const Sched *S, int n, int max_cells, cudaGraphConditionalHandle h) {
  const int ninv = S->ninv;
  cudaGraphSetConditional(h, (ninv <= max_cells && ninv < n) ? 1u : 0u);
}

// Captured partial step: an if/else graph node after the step's lists are
// built, whose branches are the persistent rung kernel (fvm_fused.cu) and
// the stage kernels; the choice is made on the device, by the step's
// involved-cell count.  Both branches give the same bits.
static int enq_fused_or_stages(fvm_ctx *c) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  k_fused_choose<<<1, 1, 0, c->st>>>(c->d.S, c->n, c->fused_max, h);
  LAUNCH_CHECK();
  CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 2;
  cudaGraphNode_t cn;
  CK(cudaGraphAddNode(&cn, g, deps, nd, &cp));
  cudaGraph_t body_fused = cp.conditional.phGraph_out[0], body_stages = cp.conditional.phGraph_out[1];
  // if: the persistent kernel (one plain kernel node), captured from the
  // auxiliary stream
  CK(cudaStreamBeginCaptureToGraph(c->aux, body_fused, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  const FusedStep a = {c->P, c->d, c->lb, c->n, c->nf, c->gbar, c->gerr};
  const cudaError_t le = fused_step_enqueue(a, c->fp32, std::min(c->fused_bpsm, FVM_FUSED_BPSM) * c->sms, c->aux);
  cudaGraph_t done = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(c->aux, &done);
  CK(le);
  CK(ee);
  c->launches += 1;
  // else: the stage kernels, captured with the auxiliary stream standing in
  // for the context's (the adjust_timesteps WHILE node nests in this branch)
  std::swap(c->st, c->aux);
  const cudaError_t be =
      cudaStreamBeginCaptureToGraph(c->st, body_stages, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  int rc = 0;
  cudaError_t ee2 = cudaSuccess;
  if (be == cudaSuccess) {
    rc = enq_stages(c, 0);
    ee2 = cudaStreamEndCapture(c->st, &done);
  }
  std::swap(c->st, c->aux);
  CK(be);
  if (rc) return rc;
  CK(ee2);
  CK(cudaStreamUpdateCaptureDependencies(c->st, &cn, 1, cudaStreamSetCaptureDependencies));
  return 0;
}

static int enq_step(fvm_ctx *c, int shared) {
  int rc;
  c->use_flist = shared ? 0 : 1;  // a global step activates every face
  if ((rc = enq_begin(c))) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->st, &cs));
  const bool fusable = !shared && c->fused_max > 0 && c->fused_bpsm > 0 && c->learn_mode == 0 && !c->reduce;
  if (fusable && cs == cudaStreamCaptureStatusActive && !c->prof) {
    rc = enq_fused_or_stages(c);
  } else if (fusable && cs == cudaStreamCaptureStatusNone) {
    // an eager step makes the same choice on the host, from the involved-cell
    // count the step's list building left on the device
    int ninv = 0;
    CK(cudaMemcpyAsync(&ninv, &c->d.S->ninv, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (ninv <= c->fused_max && ninv < c->n) {
      kt_begin(c, KT_FUSED);
      const FusedStep a = {c->P, c->d, c->lb, c->n, c->nf, c->gbar, c->gerr};
      CK(fused_step_enqueue(a, c->fp32, std::min(c->fused_bpsm, FVM_FUSED_BPSM) * c->sms, c->st));
      c->launches += 1;
      kt_end(c, KT_FUSED);
      rc = 0;
    } else {
      rc = enq_stages(c, shared);
    }
  } else {
    rc = enq_stages(c, shared);
  }
  if (rc) return rc;
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

// A grid barrier of the persistent rung kernel that gave up (the step's
// results are then incomplete): reported, and the barrier cleared.
static int check_fused_errors(fvm_ctx *c) {
  if (c->fused_max <= 0) return 0;
  int gerr = 0;
  CK(cudaMemcpy(&gerr, c->gerr, sizeof(int), cudaMemcpyDeviceToHost));
  if (!gerr) return 0;
  cudaMemset(c->gbar, 0, 2 * sizeof(unsigned));
  cudaMemset(c->gerr, 0, sizeof(int));
  c->err = "a grid barrier of the persistent rung kernel timed out";
  return FVM_ECUDA;
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
  if ((rc = check_fused_errors(c))) return rc;
  kt_collect(c);
  cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
  c->max_rung = c->hS.iscal[0];
  if ((rc = check_sched_errors(c))) return rc;
  return c->hS.iscal[1];
}

// fvm_set_state + fvm_step + fvm_get_state in one call, the host arrays read
// and then overwritten in place, with the copies of U and dU on a second
// stream overlapping the stage kernels: in before the compute_update cell
// pass needs them, out as soon as that pass has finished them (the later
// stages do not write U or dU), then the velocities after compute_pvel and
// tlast after the rungs; rung, tend and the reconstruction after the step.
// Always the stage kernels.
int fvm_step_host(fvm_ctx *c, int shared, unsigned long long tsys_ticks, double *vel, double *tlast, double *tend,
                  int *rung, double *U, double *dU, double *wrec) {
  if (!c || !c->have_mesh) return FVM_ENOMESH;
  if (!c->have_geom) { c->err = "fvm_step_host: no generator positions for this mesh (fvm_set_positions)"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_step_host: inside a step"; return FVM_EINVAL; }
  if (!vel || !tlast || !tend || !rung || !U || !dU || !wrec) {
    c->err = "fvm_step_host: every state array is required";
    return FVM_EINVAL;
  }
  for (int i = 0; i < c->n; i++)  // as fvm_set_state: nothing is uploaded when a rung is out of range
    if (rung[i] < 0 || rung[i] >= RUNGMAX - 1) { c->err = "fvm_step_host: rung out of range"; return FVM_ERANGE; }
  CK(cudaSetDevice(c->device));
  if (!c->cpy) {
    CK(cudaStreamCreateWithFlags(&c->cpy, cudaStreamNonBlocking));
    for (cudaEvent_t &e : c->hev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  Dev &d = c->d;
  const size_t n = c->n;
  cudaStream_t st = c->st, cs = c->cpy;
  const size_t wbytes = 50 * n * sizeof(double);
  double *wtmp = nullptr;  // the FP32 bulk path converts the reconstruction on the device
  // the inputs the first stages read, on the compute stream
  CK(cudaEventRecord(c->ev0, st));
  CK(cudaMemcpyAsync(d.rung, rung, n * sizeof(int), cudaMemcpyHostToDevice, st));
  if (!c->fp32) {
    CK(cudaMemcpyAsync(d.Wrec, wrec, wbytes, cudaMemcpyHostToDevice, st));
  } else {
    CK(cudaMallocAsync(&wtmp, wbytes, st));
    CK(cudaMemcpyAsync(wtmp, wrec, wbytes, cudaMemcpyHostToDevice, st));
    k_convert<double, float><<<nblk(50LL * n, 256), 256, 0, st>>>(50LL * n, wtmp, (float *)d.Wrec);
    LAUNCH_CHECK();
  }
  CK(cudaMemcpyAsync(d.tlast, tlast, n * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d.vel, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d.tend, tend, n * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d.volp, d.cvol, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  k_sched_set<<<1, 1, 0, st>>>(c->P, d.S, tsys_ticks, 0);
  LAUNCH_CHECK();
  int rc = enqueue_maxrung(c);
  if (rc) return rc;
  // U and dU on the copy stream once the early inputs are in (the two would
  // only share the link), while the step's first stages run
  CK(cudaEventRecord(c->hev[0], st));
  CK(cudaStreamWaitEvent(cs, c->hev[0], 0));
  CK(cudaMemcpyAsync(d.U, U, 10 * n * sizeof(double), cudaMemcpyHostToDevice, cs));
  CK(cudaMemcpyAsync(d.dU, dU, 14 * n * sizeof(double), cudaMemcpyHostToDevice, cs));
  CK(cudaEventRecord(c->hev[1], cs));
  c->use_flist = shared ? 0 : 1;
  if ((rc = enq_begin(c))) return rc;
  if ((rc = enq_limiter(c))) return rc;
  // the learned flux's positivity gate reads the cells' U in the flux pass
  if (c->learn_mode == 1) CK(cudaStreamWaitEvent(st, c->hev[1], 0));
  if ((rc = enq_corr_flux(c))) return rc;
  CK(cudaStreamWaitEvent(st, c->hev[1], 0));
  if ((rc = enq_corr_cell(c))) return rc;
  CK(cudaEventRecord(c->hev[2], st));
  CK(cudaStreamWaitEvent(cs, c->hev[2], 0));
  CK(cudaMemcpyAsync(U, d.U, 10 * n * sizeof(double), cudaMemcpyDeviceToHost, cs));
  CK(cudaMemcpyAsync(dU, d.dU, 14 * n * sizeof(double), cudaMemcpyDeviceToHost, cs));
  if ((rc = enq_pvel(c))) return rc;
  CK(cudaEventRecord(c->hev[3], st));
  CK(cudaStreamWaitEvent(cs, c->hev[3], 0));
  CK(cudaMemcpyAsync(vel, d.vel, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, cs));
  if ((rc = enq_timesteps(c, shared))) return rc;
  CK(cudaEventRecord(c->hev[4], st));
  CK(cudaStreamWaitEvent(cs, c->hev[4], 0));
  CK(cudaMemcpyAsync(tlast, d.tlast, n * sizeof(double), cudaMemcpyDeviceToHost, cs));
  if ((rc = enq_collect(c))) return rc;
  if ((rc = enq_update0(c))) return rc;
  if ((rc = enq_recon(c))) return rc;
  if ((rc = enq_end(c, shared))) return rc;
  CK(cudaMemcpyAsync(rung, d.rung, n * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(tend, d.tend, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (!c->fp32) {
    CK(cudaMemcpyAsync(wrec, d.Wrec, wbytes, cudaMemcpyDeviceToHost, st));
  } else {
    k_convert<float, double><<<nblk(50LL * n, 256), 256, 0, st>>>(50LL * n, (const float *)d.Wrec, wtmp);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(wrec, wtmp, wbytes, cudaMemcpyDeviceToHost, st));
    CK(cudaFreeAsync(wtmp, st));
  }
  CK(cudaEventRecord(c->ev1, st));
  CK(cudaStreamSynchronize(cs));
  c->have_state = true;
  if ((rc = read_sched(c))) return rc;
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
  if (c->reduce) { c->err = "fvm_run: a timestep reduction is installed (replayed steps cannot call the host)"; return FVM_EINVAL; }
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
  if ((rc = check_fused_errors(c))) return rc;
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
  std::vector<int> hoff(c->n + 1), hids(c->nl > 0 ? c->nl : 1);
  CK(cudaMemcpy(hoff.data(), c->d.off, sizeof(int) * (c->n + 1), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(hids.data(), c->d.lnk, sizeof(int) * c->nl, cudaMemcpyDeviceToHost));
  std::vector<unsigned char> seen(c->nf > 0 ? c->nf : 1, 0);
  int cnt = 0;
  for (int i = 0; i < c->n; i++) {
    if (!(act[i] & A_ACTIVE) || bnd[i] != NO_BOUNDARY) continue;
    for (int q = hoff[i]; q < hoff[i + 1]; q++) {
      const int f = hids[q];
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
static int mlp_launch_dev(fvm_ctx *c, int nmax, const int *n_dev, const __half *X, float *Y) {
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
                                                          c->mlp_err);
  LAUNCH_CHECK();
  return 0;
}

static int mlp_launch(fvm_ctx *c, int n, const __half *X, float *Y) {
  return mlp_launch_dev(c, n, nullptr, X, Y);
}

extern "C" {

int fvm_mlp_set_weights(fvm_ctx *c, const float *params) {
  if (!c || !params) return FVM_EINVAL;
  CK(cudaSetDevice(c->device));
  if (!c->mlp_img) {
    CK(cudaMalloc(&c->mlp_img, mlp::IMG_BYTES));
    CK(cudaMalloc(&c->mlp_err, sizeof(int)));
    CK(cudaMalloc(&c->mlp_param, mlp::NPARAM * sizeof(float)));
    CK(cudaMemsetAsync(c->mlp_err, 0, sizeof(int), c->st));
  }
  CK(cudaMemcpyAsync(c->mlp_param, params, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice, c->st));
  mlp::k_mlp_pack<<<(mlp::NH * mlp::NH + 255) / 256, 256, 0, c->st>>>(c->mlp_param, c->mlp_img);
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
  mlp::k_mlp_pack<<<(mlp::NH * mlp::NH + 255) / 256, 256, 0, c->st>>>(c->mlp_param, c->mlp_img);
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
  __half *db = nullptr;
  int *dn = nullptr;
  CK(cudaMallocAsync(&dx, nx * sizeof(float), c->st));
  CK(cudaMallocAsync(&db, nx * sizeof(__half), c->st));
  CK(cudaMallocAsync(&dy, ny * sizeof(float), c->st));
  CK(cudaMallocAsync(&dn, sizeof(int), c->st));
  CK(cudaMemcpyAsync(dx, X, nx * sizeof(float), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dy, Y, ny * sizeof(float), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(dn, &n, sizeof(int), cudaMemcpyHostToDevice, c->st));
  mlp::k_f32_to_f16<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>((long long)nx, dx, db);
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
  __half *db = nullptr;
  CK(cudaMallocAsync(&dx, nx * sizeof(float), c->st));
  CK(cudaMallocAsync(&db, nx * sizeof(__half), c->st));
  CK(cudaMallocAsync(&dy, ny * sizeof(float), c->st));
  CK(cudaMemcpyAsync(dx, X, nx * sizeof(float), cudaMemcpyHostToDevice, c->st));
  mlp::k_f32_to_f16<<<(unsigned)((nx + 255) / 256), 256, 0, c->st>>>((long long)nx, dx, db);
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

int fvm_set_flux_mode(fvm_ctx *c, int mode, float drho, float dp, float mach, float jmax, int judge, int hstride,
                      long long hcap) {
  if (!c || mode < 0 || mode > 2 || judge < 0 || hstride < 1 || hcap < 0) return FVM_EINVAL;
  if (!c->have_mesh) { c->err = "fvm_set_flux_mode: no mesh"; return FVM_ENOMESH; }
  if (mode == 1 && !c->mlp_img) { c->err = "fvm_set_flux_mode: no network weights"; return FVM_EINVAL; }
  if (!(drho >= 0.0f) || !(dp >= 0.0f) || !(mach >= 0.0f) || !(jmax >= 0.0f)) {
    c->err = "fvm_set_flux_mode: bad gate";
    return FVM_EINVAL;
  }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);
  Dev &d = c->d;
  const size_t nf = (size_t)(c->nf > 0 ? c->nf : 1);
  int rc = 0;
  if (!d.lX) {
    rc |= dalloc_bytes(c, &d.lX, nf * 16 * sizeof(__half));
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
  lb.X = (__half *)d.lX;
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
  lb.jmax = jmax;
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

long long fvm_fused_step_count(const fvm_ctx *c) { return c ? (long long)c->hS.fused_steps : -1; }

long long fvm_incremental_step_count(const fvm_ctx *c) { return c ? (long long)c->hS.inc_steps : -1; }

int fvm_set_list_building(fvm_ctx *c, int max_entries) {
  if (!c || max_entries < -1) {
    if (c) c->err = "fvm_set_list_building: max_entries must be -1 (automatic), 0 (off) or a positive bound";
    return FVM_EINVAL;
  }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);  // captured partial steps hold the choice
  c->inc_max = max_entries;
  return 0;
}

int fvm_set_reduce(fvm_ctx *c, fvm_reduce_fn fn, void *user) {
  if (!c) return FVM_EINVAL;
  if (c->in_step) { c->err = "fvm_set_reduce: inside a step"; return FVM_EINVAL; }
  c->reduce = fn;
  c->reduce_user = fn ? user : nullptr;
  return 0;
}

int fvm_set_halo(fvm_ctx *c, const unsigned char *halo) {
  if (!c || !c->have_mesh) { if (c) c->err = "fvm_set_halo: no mesh"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_set_halo: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);  // captured steps hold the parameters
  if (!halo) {
    c->P.halo = nullptr;
    return 0;
  }
  std::vector<unsigned char> h(halo, halo + c->n);
  for (auto &v : h) v = v ? 1 : 0;
  CK(cudaMemcpy(c->d.halo, h.data(), c->n, cudaMemcpyHostToDevice));
  c->P.halo = c->d.halo;
  return 0;
}

int fvm_set_fused(fvm_ctx *c, int max_cells) {
  if (!c || max_cells < 0) return FVM_EINVAL;
  if (max_cells > 0 && c->fused_bpsm <= 0) {
    c->err = "fvm_set_fused: the persistent rung kernel cannot be resident on this device";
    return FVM_EINVAL;
  }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  drop_graphs(c);  // captured partial steps hold the choice
  c->fused_max = max_cells;
  return 0;
}

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
  // the trial steps are discarded, so they take no part in a reduction over
  // ranks (one rank may tune while the others do not)
  struct ReduceOff {
    fvm_ctx *c;
    fvm_reduce_fn fn;
    ~ReduceOff() { c->reduce = fn; }
  } reduce_off{c, c->reduce};
  c->reduce = nullptr;
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
