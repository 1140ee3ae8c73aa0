// Learned face flux: a 16 -> 128 -> 128 -> 128 -> 8 GELU network that stands
// in for riemann_solver (MPI/compute_update.cpp:1109-1341) on smooth faces.
//
// Inference runs on the 5th-generation tensor cores: one CTA takes tiles of
// 128 faces; the weights sit in shared memory as FP16 in the K-major
// no-swizzle core-matrix layout the tcgen05 shared-memory descriptors
// describe; one elected thread issues tcgen05.mma (kind::f16, FP16 inputs,
// FP32 accumulation in tensor memory); each layer's bias enters the
// accumulator through one more product (a constant ONES operand times the
// bias split into two FP16 parts), so after each layer eight warps read the
// accumulator back with tcgen05.ld (32 rows x 64 columns each), apply GELU in
// packed half-precision pairs (one tanh.approx.f16x2 for two values) and
// write the next layer's FP16 A operand.  Four such tile chains
// share a CTA (one per SM) and its one copy of the weights.  The training
// products (mlp_train.cuh) keep BF16 operands.
//
// Included by fvm_kernels.cu (it uses the context and its error macros).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace mlp {

constexpr int NIN = 16, NH = 128, NOUT = 8, NOUTP = 16, TILE = 128;
constexpr int NPARAM = NH * NIN + NH + NH * NH + NH + NH * NH + NH + NOUT * NH + NOUT;
static_assert(NPARAM == 36232, "parameter count");

// byte offsets of the shared-memory image (each region 1024-byte aligned)
constexpr int KB = 16;                             // K of one tcgen05.mma of kind::f16
constexpr int OFF_W1 = 0;                          // [NH x NIN]   4096 B
constexpr int OFF_W2 = OFF_W1 + NH * NIN * 2;      // [NH x NH]   32768 B
constexpr int OFF_W3 = OFF_W2 + NH * NH * 2;       // [NH x NH]   32768 B
constexpr int OFF_W4 = OFF_W3 + NH * NH * 2;       // [NOUTP x NH] 4096 B
// Bias operands: layer L's bias is the product ONES [TILE x KB] x BL^T
// [KB x N], with columns 0 and 1 of ONES equal to 1 and of BL equal to the
// high and low FP16 parts of the bias (every other entry 0).
constexpr int OFF_B1 = OFF_W4 + NOUTP * NH * 2;    // [NH x KB]    4096 B
constexpr int OFF_B2 = OFF_B1 + NH * KB * 2;       // [NH x KB]    4096 B
constexpr int OFF_B3 = OFF_B2 + NH * KB * 2;       // [NH x KB]    4096 B
constexpr int OFF_ONES = OFF_B3 + NH * KB * 2;     // [TILE x KB]  4096 B
constexpr int OFF_B4 = OFF_ONES + TILE * KB * 2;   // [NOUTP x KB]  512 B
constexpr int IMG_BYTES = OFF_B4 + NOUTP * KB * 2;  // weights image copied from global
// GROUPS independent tile chains per CTA, each with its own activations
// buffer, mbarrier and 128 tensor-memory columns; they share the weights.
constexpr int GROUPS = 4, GTHREADS = 256;
constexpr int A_BYTES = TILE * NH * 2;             // [TILE x NH]  32768 B activations of one group
constexpr int OFF_A = (IMG_BYTES + 1023) / 1024 * 1024;  // GROUPS activations buffers
constexpr int OFF_BAR = OFF_A + GROUPS * A_BYTES;  // GROUPS mbarriers (8 B each), tensor-memory address (4 B)
constexpr int SMEM_BYTES = OFF_BAR + GROUPS * 8 + 8;
constexpr int TMEM_COLS = GROUPS * NH;             // 512: the whole tensor memory, one CTA per SM
static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");
static_assert(OFF_BAR % 8 == 0, "mbarrier alignment");
static_assert(OFF_W2 % 1024 == 0 && OFF_W3 % 1024 == 0 && OFF_W4 % 1024 == 0 && OFF_B1 % 1024 == 0 &&
                  OFF_B2 % 1024 == 0 && OFF_B3 % 1024 == 0 && OFF_ONES % 1024 == 0 && OFF_B4 % 1024 == 0 &&
                  OFF_A % 1024 == 0 && IMG_BYTES % 16 == 0,
              "align");

// Element (row, k) of a K-major no-swizzle operand with `rows` rows: core
// matrices of 8 rows x 16 bytes, 8-row groups 128 B apart (stride byte
// offset), 8-element K chunks rows/8 * 128 B apart (leading byte offset).
__host__ __device__ constexpr int kmajor_off(int row, int k, int rows) {
  return ((k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// tcgen05 shared-memory matrix descriptor, K-major, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// The same with FP16 A and B (A and B always share one type).
__host__ __device__ constexpr uint32_t instr_desc_f16(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_f16kind(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for the mbarrier phase `parity` to complete; gives up after a bounded
// number of polls and returns false.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 columns of this warp's lane quarter, with the wait in the same asm block
// (no register of the load is read before it completes).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = __uint_as_float(r[k]);
}

// The hardware tanh approximation (one MUFU instruction).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), with the
// hardware tanh in inference and training alike.
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanh_hw(u));
}

// Twice the GELU of two values, x (1 + tanh(u)) with
// u = sqrt(2/pi) x (1 + 0.044715 x^2), in packed half precision: the FP32
// sums a, b are rounded to an FP16 pair, and u, tanh and the result take one
// instruction each for both values (the pair's tanh still takes two slots of
// the XU pipe, as two FP32 tanh would).  The inference epilogue stores it and the
// image of the next layer's weights carries the factor 1/2 (an exact
// power-of-two scaling of the FP16 weights), so the layer's products are
// those of gelu(x) and W.  Past |x| = 256 the square overflows to infinity,
// tanh(u) to +-1 and the result to 2x or 0, the GELU's own limits.
__device__ __forceinline__ uint32_t gelu2_h2(float a, float b) {
  const __half2 x = __floats2half2_rn(a, b);
  const __half2 c0 = __float2half2_rn(0.7978845608028654f), c1 = __float2half2_rn(0.7978845608028654f * 0.044715f);
  const __half2 u = __hmul2(x, __hfma2(__hmul2(x, x), c1, c0));
  uint32_t t;
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t *>(&u)));
  const __half2 y = __hfma2(x, *reinterpret_cast<const __half2 *>(&t), x);
  return *reinterpret_cast<const uint32_t *>(&y);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t pack_f16(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}

// Hidden-layer epilogue of one group: warp w (0..7 within the group) takes
// rows 32 (w % 4) .. +31 (its tensor-memory lane quarter q) and columns
// 64 (w / 4) .. +63 (half h) of the group's accumulator (bias included), 32
// at a time; twice the GELU (FP16 pairs), into the group's A operand.
__device__ __forceinline__ void epilogue_hidden(uint32_t tmem, unsigned char *A, int q, int h, int lane) {
  const int r = 32 * q + lane;
#pragma unroll 1
  for (int c = 2 * h; c < 2 * h + 2; c++) {
    float v[32];
    tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * c), v);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      uint4 w;
      w.x = gelu2_h2(v[8 * j + 0], v[8 * j + 1]);
      w.y = gelu2_h2(v[8 * j + 2], v[8 * j + 3]);
      w.z = gelu2_h2(v[8 * j + 4], v[8 * j + 5]);
      w.w = gelu2_h2(v[8 * j + 6], v[8 * j + 7]);
      *reinterpret_cast<uint4 *>(A + kmajor_off(r, 32 * c + 8 * j, TILE)) = w;
    }
  }
}

// Barrier over the 256 threads of group g (named barrier 1 + g).
__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(GTHREADS) : "memory");
}
// The same barrier, returning whether v holds on every thread of the group.
__device__ __forceinline__ bool group_all(bool v, int g) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(1 + g), "r"(GTHREADS)
      : "memory");
  return r != 0;
}

// Y[n x 8] = MLP(X[n x 16]) (n read from n_dev when given); X in FP16, Y in
// FP32.  One CTA per SM (the shared memory holds one copy of the weights and
// four activations buffers); its four groups of eight warps run independent
// 128-row tiles, so one group's epilogue overlaps another's matrix products.
// The first four warps of a group load the inputs and write the outputs (warp
// q: rows 32 q .. +31); thread 0 of the group issues the group's tcgen05.mma
// and commits them to the group's mbarrier, on which the group's first warp
// waits while the other seven sleep in the group's named barrier (no polling
// that would take issue slots from the other groups' epilogues).  err bit 1:
// an mbarrier wait gave up; bit 2: the wait for that group's last commit
// before the tensor memory is released gave up as well.
constexpr int THREADS = GROUPS * GTHREADS;
static __global__ void __launch_bounds__(THREADS, 1) k_mlp_infer(int n, const int *__restrict__ n_dev,
                                                      const __half *__restrict__ X, float *__restrict__ Y,
                                                      const uint4 *__restrict__ wimg, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  if (n_dev) n = *n_dev;  // row count produced on the device
  const int t = threadIdx.x, warp = t >> 5, g = warp >> 3, q = warp & 3, hq = (warp >> 2) & 1,
            gt = t & (GTHREADS - 1);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + OFF_BAR + GROUPS * 8);
  unsigned char *A = sm + OFF_A + g * A_BYTES;
  for (int i = t; i < IMG_BYTES / 16; i += blockDim.x) reinterpret_cast<uint4 *>(sm)[i] = wimg[i];
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    for (int i = 0; i < GROUPS; i++) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bars + i)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t tmem = tbase + (uint32_t)(g * NH);  // this group's 128 columns
  const uint32_t bar_a = smem_u32(bars + g);
  const uint32_t a_addr = smem_u32(A);
  const uint32_t w_addr = smem_u32(sm);
  const uint32_t id_h = instr_desc_f16(TILE, NH), id_o = instr_desc_f16(TILE, NOUTP);
  const uint32_t LBO_128 = (128 / 8) * 128, LBO_OUT = (NOUTP / 8) * 128, SBO = 128;
  const uint64_t ones_desc = smem_desc(w_addr + OFF_ONES, LBO_128, SBO);
  uint32_t parity = 0;
  bool ok = true;
  const int ntiles = (n + TILE - 1) / TILE;
  const int stride = gridDim.x * GROUPS;
  // layer-1 input: thread gt of the group holds row gt of X (16 FP16, two
  // 16-byte halves); the next tile's row is loaded while this tile's layers run
  auto load_x = [&](int tile, uint4 &x0, uint4 &x1) {
    x0 = x1 = make_uint4(0, 0, 0, 0);
    if (tile < ntiles && gt < TILE) {
      const int row = tile * TILE + gt;
      if (row < n) {
        const uint4 *src = reinterpret_cast<const uint4 *>(X + (size_t)row * NIN);
        x0 = src[0];
        x1 = src[1];
      }
    }
  };
  int tile = blockIdx.x * GROUPS + g;
  uint4 x0, x1;
  load_x(tile, x0, x1);
  for (; tile < ntiles && ok; tile += stride) {
    if (gt < TILE) {
      *reinterpret_cast<uint4 *>(A + kmajor_off(gt, 0, TILE)) = x0;
      *reinterpret_cast<uint4 *>(A + kmajor_off(gt, 8, TILE)) = x1;
    }
    load_x(tile + stride, x0, x1);
    // four layers; each reads the group's A (and the weights) and overwrites
    // the group's accumulator, whose previous contents the group has read
#pragma unroll 1
    for (int L = 0; L < 4 && ok; L++) {
      fence_async_smem();
      fence_before();
      group_sync(g);
      if (gt == 0) {
        fence_after();
        const uint32_t lbo_b = L == 3 ? LBO_OUT : LBO_128, idesc = L == 3 ? id_o : id_h;
        // the bias first (it initialises the accumulator), then the weights
        const uint32_t bb = w_addr + (L == 0 ? OFF_B1 : L == 1 ? OFF_B2 : L == 2 ? OFF_B3 : OFF_B4);
        mma_f16kind(tmem, ones_desc, smem_desc(bb, lbo_b, SBO), idesc, 0);
        if (L == 0) {
          mma_f16kind(tmem, smem_desc(a_addr, LBO_128, SBO), smem_desc(w_addr + OFF_W1, LBO_128, SBO), id_h, 1);
        } else {
          const uint32_t wb = w_addr + (L == 1 ? OFF_W2 : L == 2 ? OFF_W3 : OFF_W4);
#pragma unroll 1
          for (int kk = 0; kk < NH / KB; kk++)
            mma_f16kind(tmem, smem_desc(a_addr + 2 * kk * LBO_128, LBO_128, SBO),
                        smem_desc(wb + 2 * kk * lbo_b, lbo_b, SBO), idesc, 1);
        }
        mma_commit(bar_a);
      }
      const bool waited = gt < 32 ? bar_wait(bar_a, parity) : true;
      if (!group_all(waited, g)) {  // the group leaves together
        if (gt == 0) atomicOr(err, 1);
        ok = false;
        break;
      }
      parity ^= 1;
      fence_after();
      if (L < 3) {
        epilogue_hidden(tmem, A, q, hq, t & 31);
      } else if (gt < TILE) {
        float v[8];
        tmem_ld8(tmem + ((uint32_t)(32 * q) << 16), v);
        const int row = tile * TILE + gt;
        if (row < n) {
          float4 *yo = reinterpret_cast<float4 *>(Y + (size_t)row * NOUT);
          yo[0] = make_float4(v[0], v[1], v[2], v[3]);
          yo[1] = make_float4(v[4], v[5], v[6], v[7]);
        }
      }
    }
  }
  // A group that gave up on its mbarrier may still have matrix products in
  // flight that write its tensor-memory columns: wait once more (bounded) for
  // that commit before the columns are released; err bit 2 records that this
  // wait gave up too (the columns are then released with the products
  // possibly still running, and the launch reports the error).
  if (!ok && !bar_wait(bar_a, parity) && gt == 0) atomicOr(err, 2);
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TMEM_COLS));
  }
}

static __global__ void k_f32_to_f16(long long n, const float *__restrict__ x, __half *__restrict__ y) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2half_rn(x[i]);
}

// Parameters (W1[NH x NIN], b1, W2[NH x NH], b2, W3, b3, W4[NOUT x NH], b4)
// -> shared-memory image: the FP16 weights (W4 padded to NOUTP rows with
// zeros), the bias operands (each bias as the FP16 pair hi = fp16(b),
// lo = fp16(b - hi), b4 padded with zeros) and the ONES operand.  W2, W3 and
// W4 are stored halved: the epilogue hands them twice the GELU.
static __global__ void k_mlp_pack(const float *__restrict__ p, unsigned char *__restrict__ img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const float *W1 = p, *b1 = W1 + NH * NIN, *W2 = b1 + NH, *b2 = W2 + NH * NH, *W3 = b2 + NH, *b3 = W3 + NH * NH,
              *W4 = b3 + NH, *b4 = W4 + NOUT * NH;
  if (i < NH * NIN) {
    const int r = i / NIN, k = i % NIN;
    *reinterpret_cast<__half *>(img + OFF_W1 + kmajor_off(r, k, NH)) = __float2half_rn(W1[i]);
  }
  if (i < NH * NH) {
    const int r = i / NH, k = i % NH;
    *reinterpret_cast<__half *>(img + OFF_W2 + kmajor_off(r, k, NH)) = __float2half_rn(0.5f * W2[i]);
    *reinterpret_cast<__half *>(img + OFF_W3 + kmajor_off(r, k, NH)) = __float2half_rn(0.5f * W3[i]);
  }
  if (i < NOUTP * NH) {
    const int r = i / NH, k = i % NH;
    *reinterpret_cast<__half *>(img + OFF_W4 + kmajor_off(r, k, NOUTP)) =
        __float2half_rn(r < NOUT ? 0.5f * W4[r * NH + k] : 0.0f);
  }
  auto bias_entry = [](float b, int k) {
    const __half hi = __float2half_rn(b);
    return k == 0 ? hi : k == 1 ? __float2half_rn(b - __half2float(hi)) : __float2half_rn(0.0f);
  };
  if (i < NH * KB) {
    const int r = i / KB, k = i % KB;
    *reinterpret_cast<__half *>(img + OFF_B1 + kmajor_off(r, k, NH)) = bias_entry(b1[r], k);
    *reinterpret_cast<__half *>(img + OFF_B2 + kmajor_off(r, k, NH)) = bias_entry(b2[r], k);
    *reinterpret_cast<__half *>(img + OFF_B3 + kmajor_off(r, k, NH)) = bias_entry(b3[r], k);
    *reinterpret_cast<__half *>(img + OFF_ONES + kmajor_off(r, k, TILE)) = __float2half_rn(k < 2 ? 1.0f : 0.0f);
  }
  if (i < NOUTP * KB) {
    const int r = i / KB, k = i % KB;
    *reinterpret_cast<__half *>(img + OFF_B4 + kmajor_off(r, k, NOUTP)) = bias_entry(r < NOUT ? b4[r] : 0.0f, k);
  }
}

}  // namespace mlp
