// Device helpers shared by the generated mechanism code and the kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

// Literal-mode select: LM == 0 keeps the reference build's literal kinds (default-real
// literals rounded to float32), LM == 1 reads every literal as a double.
#define TNG_LM(ref, dbl) (LM ? (dbl) : (ref))
// Scheduling fence for generated straight-line code: memory operations are not moved across it,
// which bounds how many loads the compiler hoists (and so the registers they hold).
#define TNG_SCHED_FENCE() asm volatile("" ::: "memory")

namespace tng {

// 2^x on the FP32 special-function unit (ex2.approx, flushes subnormal results to zero).
__device__ __forceinline__ float tng_ex2f(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// log2(x) on the FP32 special-function unit; log2(0) = -inf.
__device__ __forceinline__ float tng_lg2f(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// log2(1 + 2^x) without overflow for large x.
__device__ __forceinline__ float tng_softplus2f(float x) {
  return fmaxf(x, 0.0f) + tng_lg2f(1.0f + tng_ex2f(-fabsf(x)));
}

}  // namespace tng
