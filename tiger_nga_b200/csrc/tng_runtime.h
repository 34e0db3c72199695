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
int solver_prepare(tng_chem* h);
// NASA tables on the device (ns x 24: high range 12, low range 12) and the switch temperature
void solver_thermo(tng_chem* h, const double** th, double* tmid);
int substep_run(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts, double dt, double p,
                int flags, const int* list, const int* nlist, int* cell_nst, int* cell_nni, int* cell_status,
                tng_substep_stats* stats);

}  // namespace tng

struct tng_chem {
  const tng::MechOps* ops = nullptr;
  tng_cfg cfg{};
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream[2] = {nullptr, nullptr};
  tng::DevBuf bufs[11];  // 0-3 rate staging, 4-5 solver, 6-7 Fortran substep, 8-9 mixture properties, 10 shims
  tng::SolverState* solver = nullptr;
  int dependents = 0;  // live tng_mlp / tng_surrogate objects using this handle's stream
  double props_inv_lewis[64];  // reciprocal Lewis numbers held in bufs[8] (props_lewis_n of them)
  int props_lewis_n = 0;
};
