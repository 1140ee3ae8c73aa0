// Training kernels of the learned face flux (the network of flux_mlp.cuh):
// forward and backward passes built from one strided BF16 tensor-core GEMM
// (mma.sync m16n8k16, FP32 accumulation), elementwise bias/GELU kernels, a
// mean-squared loss and Adam.  Activations are stored in FP32 holding
// BF16-rounded values, weights as an FP32 master copy rounded to BF16 where
// they enter a product, as in inference.
//
// Included by fvm_kernels.cu.

namespace mlpt {

using mlp::NIN;
using mlp::NH;
using mlp::NOUT;
using mlp::NPARAM;

// C[m, n] (+)= sum_k A(m, k) B(k, n), A(m, k) = A[m*sam + k*sak],
// B(k, n) = B[k*sbk + n*sbn], C row-major with leading dimension ldc.
// 64 x 64 tiles, K in steps of 16, four warps of 32 x 32.
constexpr int GT = 64, GK = 16;

__device__ __forceinline__ uint32_t pk(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const float *__restrict__ A, long long sam,
                                              long long sak, const float *__restrict__ B, long long sbk,
                                              long long sbn, float *__restrict__ C, int ldc, int accumulate) {
  __shared__ __nv_bfloat16 As[GT][GK + 8];   // [m][k]
  __shared__ __nv_bfloat16 Bs[GT][GK + 8];   // [n][k]
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
  const int wm = (w >> 1) * 32, wn = (w & 1) * 32;
  const int g = lane >> 2, q = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[i][j][r] = 0.0f;
  for (int k0 = 0; k0 < K; k0 += GK) {
    // 64 x 16 elements of each operand, 8 per thread
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int idx = t + 128 * e, r = idx >> 4, k = idx & 15;
      const int gm = m0 + r, gn = n0 + r, gk = k0 + k;
      const float av = (gm < M && gk < K) ? A[gm * sam + gk * sak] : 0.0f;
      const float bv = (gn < N && gk < K) ? B[gk * sbk + gn * sbn] : 0.0f;
      As[r][k] = __float2bfloat16_rn(av);
      Bs[r][k] = __float2bfloat16_rn(bv);
    }
    __syncthreads();
    uint32_t af[2][4], bf[4][2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int r = wm + 16 * i + g;
      af[i][0] = pk(As[r][2 * q], As[r][2 * q + 1]);
      af[i][1] = pk(As[r + 8][2 * q], As[r + 8][2 * q + 1]);
      af[i][2] = pk(As[r][2 * q + 8], As[r][2 * q + 9]);
      af[i][3] = pk(As[r + 8][2 * q + 8], As[r + 8][2 * q + 9]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = wn + 8 * j + g;
      bf[j][0] = pk(Bs[c][2 * q], Bs[c][2 * q + 1]);
      bf[j][1] = pk(Bs[c][2 * q + 8], Bs[c][2 * q + 9]);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
            "{%0, %1, %2, %3};"
            : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
            : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bf[j][0]), "r"(bf[j][1]));
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int gm = m0 + wm + 16 * i + g + (r >= 2 ? 8 : 0);
        const int gn = n0 + wn + 8 * j + 2 * q + (r & 1);
        if (gm < M && gn < N) {
          float *cp = C + (size_t)gm * ldc + gn;
          *cp = accumulate ? *cp + acc[i][j][r] : acc[i][j][r];
        }
      }
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
