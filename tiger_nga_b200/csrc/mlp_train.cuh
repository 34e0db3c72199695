// K5/K6: training kernels of the surrogate MLP (FP32): tiled GEMMs with fused bias/GELU
// epilogues, GELU backward, loss gradient, bias gradient, split-K weight-gradient reduction and
// Adam. Deterministic: no floating-point atomics.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace tng {

constexpr float kGeluC0 = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float kGeluC1 = 0.044715f;

__device__ __forceinline__ float gelu_f(float x) {
  return 0.5f * x * (1.0f + tanhf(kGeluC0 * (x + kGeluC1 * x * x * x)));
}

__device__ __forceinline__ float gelu_grad_f(float x) {
  const float u = kGeluC0 * (x + kGeluC1 * x * x * x);
  const float th = tanhf(u);
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * kGeluC0 * (1.0f + 3.0f * kGeluC1 * x * x);
}

// C[M x N] = op(A)[M x K] * op(B)[K x N]
//   op(A)[m][k] = TA ? A[k*lda + m] : A[m*lda + k]
//   op(B)[k][n] = TB ? B[n*ldb + k] : B[k*ldb + n]
// EPI 0: C = acc;  1: C = acc + bias[n];  2: P = acc + bias[n], C = gelu(P).
// Split-K: blockIdx.z covers K range [z*kchunk, (z+1)*kchunk); C is offset by z*M*ldc.
constexpr int kBM = 64, kBN = 64, kBK = 16;

template <int TA, int TB, int EPI>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                               const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                               const float* __restrict__ bias, float* __restrict__ P, int kchunk) {
  __shared__ float As[kBK][kBM + 4];
  __shared__ float Bs[kBK][kBN + 4];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(K, kb + kchunk);
  C += (size_t)blockIdx.z * M * ldc;
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += kBK) {
    // 64 x 16 tile of op(A) and 16 x 64 tile of op(B): 1024 elements each, 4 per thread
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int e = tid + 256 * i;
      int mm, kk;
      if (TA) {
        mm = e & 63;
        kk = e >> 6;
      } else {
        kk = e & 15;
        mm = e >> 4;
      }
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.f;
      if (gm < M && gk < ke) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
      As[kk][mm] = v;
      int nn;
      if (TB) {
        kk = e & 15;
        nn = e >> 4;
      } else {
        nn = e & 63;
        kk = e >> 6;
      }
      const int gn = n0 + nn;
      const int gk2 = k0 + kk;
      float u = 0.f;
      if (gn < N && gk2 < ke) u = TB ? B[(size_t)gn * ldb + gk2] : B[(size_t)gk2 * ldb + gn];
      Bs[kk][nn] = u;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty * 4 + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx * 4 + j;
      if (gn >= N) continue;
      float v = acc[i][j];
      if (EPI >= 1) v += bias[gn];
      if (EPI == 2) {
        P[(size_t)gm * ldc + gn] = v;
        v = gelu_f(v);
      }
      C[(size_t)gm * ldc + gn] = v;
    }
  }
}

// dZ = dH * gelu'(P)
__global__ void k_gelu_back(const float* __restrict__ dH, const float* __restrict__ P, float* __restrict__ dZ,
                            int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dZ[i] = dH[i] * gelu_grad_f(P[i]);
}

// Loss sum_o w_o a(r) (y - t)^2 / (rows * nout), a(r) = under for r = y - t < 0 and 1 otherwise,
// and its gradient; per-block partial sums of the loss.
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ w, int rows,
                      int nout, int ld, float under, float* __restrict__ dY, float* __restrict__ partial) {
  __shared__ float red[256];
  float s = 0.f;
  const float scale = 1.0f / ((float)rows * (float)nout);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)rows * ld;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int o = (int)(e % ld);
    const float r = Y[e] - T[e];
    const float wo = o < nout ? (r < 0.f ? under * w[o] : w[o]) : 0.f;
    s += wo * r * r;
    dY[e] = 2.f * wo * r * scale;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0] * scale;
}

// db[n] = sum over rows of dZ[r][n] (one thread per column, fixed order)
__global__ void k_colsum(const float* __restrict__ dZ, int rows, int n, int ld, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += dZ[(size_t)r * ld + c];
  db[c] = s;
}

// out[i] = sum_z part[z*n + i]  (split-K reduction, fixed order)
__global__ void k_sum_parts(const float* __restrict__ part, int nz, int64_t n, float* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int z = 0; z < nz; ++z) s += part[(size_t)z * n + i];
    out[i] = s;
  }
}

// Adam with bias correction; bc1 = 1 - b1^t, bc2 = 1 - b2^t
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// rows of src selected by idx -> dst (row length ld)
__global__ void k_gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int rows, int ld,
                              float* __restrict__ dst) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)rows * ld;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / ld), c = (int)(e % ld);
    dst[e] = src[(size_t)idx[r] * ld + c];
  }
}

}  // namespace tng
