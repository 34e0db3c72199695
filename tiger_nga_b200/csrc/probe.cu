// Measurement helper: sustained FP64 FMA throughput of the device, the denominator of the
// FP64-pipe roofline reported next to the rate kernels.
#include <cuda_runtime.h>

#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

__global__ void __launch_bounds__(256) k_dfma_peak(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 123.456) out[blockIdx.x] = s;  // keeps the chains live; never true for these inputs
}

}  // namespace tng

extern "C" int tng_bench_fp64_peak(int device, double* tflops) {
  using namespace tng;
  if (!tflops) return set_error(TNG_ERR_ARG, "tng_bench_fp64_peak: null output");
  DeviceGuard g(device);
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceProperties");
  double* out = nullptr;
  if ((e = cudaMalloc(&out, sizeof(double) * 65536)) != cudaSuccess) return cuda_error(e, "cudaMalloc");
  const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_dfma_peak<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(a);
  k_dfma_peak<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(b);
  e = cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_error(e, "fp64 peak kernel");
  const double flops = 2.0 * 64.0 * iters * (double)blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return TNG_OK;
}
