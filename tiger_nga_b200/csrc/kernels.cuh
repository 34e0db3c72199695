// Rate-evaluation kernels and the per-mechanism operation table (sm_100a).
//
// K1: batched finitechem_compute_rhs (combustion/finitechem.f90:93-175) with the mechanism's
// PRODRATES / GETLINDRATECOEFF / COMPTHERMODATA generated as straight-line device code.
// One cell per thread; the state is species-major (variable v of cell i at [v*ld + i]), so
// each of the N+1 loads and stores of a warp touches one contiguous 256-byte segment.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tng_device.cuh"

namespace tng {

constexpr int kRhsMaxBlock = 256;

template <class Mech, int LM, int PREC, bool DUMP>
__global__ void __launch_bounds__(kRhsMaxBlock) k_rhs(const double* __restrict__ sol, double* __restrict__ out,
                                                      double* __restrict__ dump, long long n, long long ld, double p) {
  constexpr int NV = Mech::NS + 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double s[NV], r[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = __ldcs(sol + v * ld + i);
    if constexpr (PREC == 0)
      Mech::template rhs_fp64<LM, DUMP>(s, p, r, DUMP ? dump + i : nullptr, ld);
    else
      Mech::template rhs_mixed<LM, DUMP>(s, p, r, DUMP ? dump + i : nullptr, ld);
#pragma unroll
    for (int v = 0; v < NV; ++v) __stcs(out + v * ld + i, r[v]);
  }
}

// Launch geometry for the grid-stride rate kernel: one thread per cell up to a cap of
// 64 resident blocks' worth per SM (the loop covers the rest).
inline unsigned rhs_grid(long long n, int block) {
  long long b = (n + block - 1) / block;
  long long cap = 148LL * 64;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

struct MechOps {
  const char* name;
  int ns, nslot, nm, nelem;
  const char* const* species;
  const double* wmol[2];
  const char* const* elements;
  const double* elem;  // nelem x ns, row-major
  // rate evaluation: prec 0/1, lm 0/1; dump may be null
  cudaError_t (*rhs)(int prec, int lm, const double* sol, double* out, double* dump, long long n, long long ld,
                     double p, int block, cudaStream_t st);
};

template <class Mech>
cudaError_t launch_rhs(int prec, int lm, const double* sol, double* out, double* dump, long long n, long long ld,
                       double p, int block, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (block <= 0 || block > kRhsMaxBlock) block = 128;
  const unsigned grid = rhs_grid(n, block);
  const bool d = dump != nullptr;
  if (prec == 0) {
    if (lm == 0) {
      if (d)
        k_rhs<Mech, 0, 0, true><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
      else
        k_rhs<Mech, 0, 0, false><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
    } else {
      if (d) return cudaErrorInvalidValue;
      k_rhs<Mech, 1, 0, false><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
    }
  } else {
    if (lm == 0) {
      if (d)
        k_rhs<Mech, 0, 1, true><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
      else
        k_rhs<Mech, 0, 1, false><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
    } else {
      if (d) return cudaErrorInvalidValue;
      k_rhs<Mech, 1, 1, false><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
    }
  }
  return cudaGetLastError();
}

}  // namespace tng
