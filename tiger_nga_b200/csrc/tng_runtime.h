// Host runtime internals shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "kernels.cuh"
#include "tiger_chem.h"

struct tng_chem;

namespace tng {

int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);

// Null-terminated list of the built-in mechanisms (generated registry).
const MechOps* const* all_mechanisms();

// Makes a device current for the scope and restores the caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Grow-only device buffer owned by a handle.
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  bool reserve(size_t bytes) {
    if (bytes <= cap) return true;
    release();
    if (cudaMalloc(&ptr, bytes) != cudaSuccess) {
      ptr = nullptr;
      return false;
    }
    cap = bytes;
    return true;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

struct SolverState;
void solver_release(tng_chem* h);

}  // namespace tng

struct tng_chem {
  const tng::MechOps* ops = nullptr;
  tng_cfg cfg{};
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream[2] = {nullptr, nullptr};
  tng::DevBuf bufs[8];
  tng::SolverState* solver = nullptr;
};
