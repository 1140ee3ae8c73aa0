// Training kernels of the learned face flux (the network of flux_mlp.cuh):
// forward and backward passes built from one strided BF16 tensor-core GEMM
// (tcgen05.mma, FP32 accumulation in tensor memory), elementwise bias/GELU
// kernels, a mean-squared loss and Adam.  Activations are stored in FP32 holding
// BF16-rounded values, weights as an FP32 master copy rounded to BF16 where
// they enter a product, as in inference.
//
// Included by fvm_kernels.cu.
#pragma once

namespace mlpt {

using mlp::NIN;
using mlp::NH;
using mlp::NOUT;
using mlp::NPARAM;

// C[m, n] (+)= sum_k A(m, k) B(k, n), A(m, k) = A[m*sam + k*sak],
// B(k, n) = B[k*sbk + n*sbn], C row-major with leading dimension ldc: every
// product of the forward and backward passes, on the 5th-generation tensor
// cores.  One CTA (four warps) owns a 128 x 128 tile of C in 128 columns of
// tensor memory (FP32).  K runs in chunks of 64 through two shared-memory
// stages: all threads load a chunk of each operand from global memory with
// the operand's strides (so transposed operands need no copy), round it to
// BF16 and store it in the K-major no-swizzle core-matrix layout; one thread
// issues four tcgen05.mma (kind::f16, K = 16 each) on it and commits them to
// the stage's mbarrier, which the chunk two steps later waits on before it
// overwrites the stage.  Rows, columns and K past the operand's extent are
// zero-filled.  With gridDim.z > 1 the K range is split: split z covers
// chunks [z*cps, (z+1)*cps) and writes its partial tile to
// Cpart[z][M][N] (reduced in a fixed order by k_splitk_sum), so the weight
// gradients (M, N <= 128, K = batch rows) spread over many SMs and stay
// deterministic.  err bit 4: an mbarrier wait gave up.
constexpr int TM = 128, TN = 128, TK = 64;
constexpr int TC_A = TM * TK * 2, TC_B = TN * TK * 2;  // bytes of one stage's operand tiles
constexpr int TC_SMEM = 2 * (TC_A + TC_B) + 32;          // two stages, two mbarriers, tensor-memory slot

// One operand tile (rows x TK, `rows` = TM or TN) of chunk k0 into shared
// memory: element (r, k) = P[(base + r) * s_row + (k0 + k) * s_k], rounded to
// BF16, zero outside rows < nrows and k < K.  The index order follows the
// operand's unit stride, and where that stride is 1 and every run of four
// starts on a 16-byte boundary the loads are float4: along K four elements
// go out as one 8-byte store of two BF16 pairs (they are adjacent in a core
// matrix row), along the rows as four 2-byte stores.
template <int ROWS>
__device__ __forceinline__ void tc_load_operand(unsigned char *sdst, int base, int nrows, int k0, int K,
                                                const float *__restrict__ P, long long s_row, long long s_k) {
  const int t = threadIdx.x;
  const bool kvec = s_k == 1 && (s_row & 3) == 0 && (K & 3) == 0 && (reinterpret_cast<uintptr_t>(P) & 15) == 0;
  const bool rvec = s_row == 1 && (s_k & 3) == 0 && (nrows & 3) == 0 && (base & 3) == 0 &&
                    (reinterpret_cast<uintptr_t>(P) & 15) == 0;
  if (kvec) {
#pragma unroll 4
    for (int e = t; e < ROWS * TK / 4; e += 128) {
      const int r = e / (TK / 4), k = (e % (TK / 4)) * 4;
      const int gr = base + r, gk = k0 + k;
      float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (gr < nrows && gk < K) v = *reinterpret_cast<const float4 *>(P + gr * s_row + gk);
      uint2 w;
      w.x = mlp::pack_bf16(v.x, v.y);
      w.y = mlp::pack_bf16(v.z, v.w);
      *reinterpret_cast<uint2 *>(sdst + mlp::kmajor_off(r, k, ROWS)) = w;
    }
  } else if (rvec) {
#pragma unroll 4
    for (int e = t; e < ROWS * TK / 4; e += 128) {
      const int r = (e % (ROWS / 4)) * 4, k = e / (ROWS / 4);
      const int gr = base + r, gk = k0 + k;
      float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (gr < nrows && gk < K) v = *reinterpret_cast<const float4 *>(P + gr + gk * s_k);
      const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int q = 0; q < 4; q++)
        *reinterpret_cast<__nv_bfloat16 *>(sdst + mlp::kmajor_off(r + q, k, ROWS)) = __float2bfloat16_rn(vv[q]);
    }
  } else {
#pragma unroll 4
    for (int e = t; e < ROWS * TK; e += 128) {
      const int r = s_k == 1 ? e / TK : e % ROWS, k = s_k == 1 ? e % TK : e / ROWS;
      const int gr = base + r, gk = k0 + k;
      const float v = (gr < nrows && gk < K) ? P[gr * s_row + gk * s_k] : 0.0f;
      *reinterpret_cast<__nv_bfloat16 *>(sdst + mlp::kmajor_off(r, k, ROWS)) = __float2bfloat16_rn(v);
    }
  }
}

__device__ __forceinline__ void tc_load_stage(unsigned char *sa, unsigned char *sb, int m0, int n0, int k0, int M,
                                              int N, int K, const float *__restrict__ A, long long sam,
                                              long long sak, const float *__restrict__ B, long long sbk,
                                              long long sbn) {
  tc_load_operand<TM>(sa, m0, M, k0, K, A, sam, sak);  // A(m, k) = A[m sam + k sak]
  tc_load_operand<TN>(sb, n0, N, k0, K, B, sbn, sbk);  // B(k, n) = B[k sbk + n sbn], as rows n
}

__global__ void __launch_bounds__(128) k_gemm_tc(int M, int N, int K, const float *__restrict__ A, long long sam,
                                                 long long sak, const float *__restrict__ B, long long sbk,
                                                 long long sbn, float *__restrict__ C, int ldc, int accumulate,
                                                 int cps, float *__restrict__ Cpart, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *sa[2] = {sm, sm + TC_A + TC_B};
  unsigned char *sb[2] = {sm + TC_A, sm + 2 * TC_A + TC_B};
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + 2 * (TC_A + TC_B));
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const int nchunk_all = (K + TK - 1) / TK;
  const int c_begin = gridDim.z > 1 ? blockIdx.z * cps : 0;
  const int c_end = gridDim.z > 1 ? min(nchunk_all, c_begin + cps) : nchunk_all;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(mlp::smem_u32(tslot)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    for (int i = 0; i < 2; i++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mlp::smem_u32(bars + i)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  mlp::fence_before();
  __syncthreads();
  mlp::fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = mlp::instr_desc(TM, TN);
  constexpr uint32_t LBO_A = (TM / 8) * 128, LBO_B = (TN / 8) * 128, SBO = 128;
  bool ok = true;
  int issued = 0;  // chunks whose products were issued and committed
  for (int ch = c_begin; ch < c_end && ok; ch++) {
    const int st = (ch - c_begin) & 1, use = (ch - c_begin) >> 1;
    if (use > 0) {  // the products of this stage's previous chunk have read it
      const bool w = mlp::bar_wait(mlp::smem_u32(bars + st), (uint32_t)((use - 1) & 1));
      if (!__syncthreads_and(w)) { ok = false; break; }
    }
    tc_load_stage(sa[st], sb[st], m0, n0, ch * TK, M, N, K, A, sam, sak, B, sbk, sbn);
    mlp::fence_async_smem();
    mlp::fence_before();
    __syncthreads();
    if (t == 0) {
      mlp::fence_after();
      const uint32_t a = mlp::smem_u32(sa[st]), b = mlp::smem_u32(sb[st]);
#pragma unroll
      for (int kk = 0; kk < TK / 16; kk++)
        mlp::mma_f16kind(tmem, mlp::smem_desc(a + 2 * kk * LBO_A, LBO_A, SBO), mlp::smem_desc(b + 2 * kk * LBO_B, LBO_B, SBO),
                      idesc, (ch > c_begin || kk > 0) ? 1u : 0u);
      mlp::mma_commit(mlp::smem_u32(bars + st));
    }
    issued++;
  }
  const int nch = c_end - c_begin;
  if (ok && nch > 0) {  // the last commit covers every product issued before it
    const int st = (nch - 1) & 1, use = (nch - 1) >> 1;
    ok = __syncthreads_and(mlp::bar_wait(mlp::smem_u32(bars + st), (uint32_t)(use & 1)));
  }
  if (!ok) {
    if (t == 0) atomicOr(err, 4);
    // a stage may still have products in flight: wait (bounded) for each
    // stage's last issued commit before the tensor memory is released
    for (int st = 0; st < 2 && st < issued; st++) {
      const int last_use = (issued - 1 - st) >> 1;
      mlp::bar_wait(mlp::smem_u32(bars + st), (uint32_t)(last_use & 1));
    }
  } else {
    mlp::fence_after();
    const int row = m0 + 32 * warp + lane;
#pragma unroll 1
    for (int cb = 0; cb < TN && n0 + cb < N; cb += 32) {
      float v[32];
      if (nch > 0) {
        mlp::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)cb, v);
      } else {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] = 0.0f;
      }
      if (row < M) {
        if (gridDim.z > 1) {
          float *o = Cpart + ((size_t)blockIdx.z * M + row) * N + n0 + cb;
#pragma unroll
          for (int j = 0; j < 32; j++)
            if (n0 + cb + j < N) o[j] = v[j];
        } else {
          float *o = C + (size_t)row * ldc + n0 + cb;
#pragma unroll
          for (int j = 0; j < 32; j++)
            if (n0 + cb + j < N) o[j] = accumulate ? o[j] + v[j] : v[j];
        }
      }
    }
  }
  mlp::fence_before();
  __syncthreads();
  if (warp == 0) {
    mlp::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
  }
}

// C[m, n] (+)= sum over splits of Cpart[z][m][n], in split order.
__global__ void k_splitk_sum(int M, int N, int nsplit, const float *__restrict__ Cpart, float *__restrict__ C,
                             int ldc, int accumulate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  float s = 0.0f;
  for (int z = 0; z < nsplit; z++) s += Cpart[(size_t)z * M * N + i];
  float *o = C + (size_t)(i / N) * ldc + i % N;
  *o = accumulate ? *o + s : s;
}

// Z += b (pre-activation kept), A = BF16(GELU(Z)).
__global__ void k_bias_gelu(int rows, int cols, float *__restrict__ Z, const float *__restrict__ b,
                            float *__restrict__ A) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)rows * cols) return;
  const float z = Z[i] + b[i % cols];
  Z[i] = z;
  A[i] = __bfloat162float(__float2bfloat16_rn(mlp::gelu(z)));
}

// Output layer: Y = Z + b; G = dL/dY of L = mean w (Y - T)^2; loss summed.
__global__ void k_out_loss(int rows, const float *__restrict__ Z, const float *__restrict__ b,
                           const float *__restrict__ T, const float *__restrict__ wt, float *__restrict__ G,
                           float *__restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (i < rows * NOUT) {
    const int k = i % NOUT;
    const float r = Z[i] + b[k] - T[i];
    const float s = 1.0f / (float)(rows * NOUT);
    G[i] = 2.0f * wt[k] * r * s;
    l = wt[k] * r * r * s;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

__device__ __forceinline__ float gelu_grad(float x) {
  const float c = 0.7978845608028654f;
  const float t = mlp::tanh_hw(c * (x + 0.044715f * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * c * (1.0f + 3.0f * 0.044715f * x * x);
}

// dZ = dA * GELU'(Z), in place on dA.
__global__ void k_gelu_back(long long n, float *__restrict__ dA, const float *__restrict__ Z) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dA[i] *= gelu_grad(Z[i]);
}

// db[c] = sum over rows of dZ[r, c] (one thread per column, fixed order).
__global__ void k_colsum(int rows, int cols, const float *__restrict__ dZ, float *__restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; r++) s += dZ[(size_t)r * cols + c];
  db[c] = s;
}

__global__ void k_adam(int n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Minibatch rows drawn with a counter-based hash of (seed, step, row).
__global__ void k_gather(long long n, const float *__restrict__ X, const float *__restrict__ T, int rows,
                         unsigned long long seed, int step, float *__restrict__ bX, float *__restrict__ bT) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const long long src = (long long)(mix64(seed ^ ((unsigned long long)step << 32) ^ (unsigned long long)r) %
                                    (unsigned long long)n);
#pragma unroll
  for (int k = 0; k < NIN; k++) bX[(size_t)r * NIN + k] = X[src * NIN + k];
#pragma unroll
  for (int k = 0; k < NOUT; k++) bT[(size_t)r * NOUT + k] = T[src * NOUT + k];
}

}  // namespace mlpt
