// Rate-evaluation kernels and the per-mechanism operation table (sm_100a).
//
// K1: batched finitechem_compute_rhs (combustion/finitechem.f90:93-175) with the mechanism's
// PRODRATES / GETLINDRATECOEFF / COMPTHERMODATA generated as straight-line device code.
// One cell per thread; the state is species-major (variable v of cell i at [v*ld + i]), so
// each of the N+1 loads and stores of a warp touches one contiguous 256-byte segment.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "solver_layout.h"
#include "tng_device.cuh"

namespace tng {

constexpr int kRhsMaxBlock = 256;

// SYNC != 0 inserts block barriers every 48 slots inside the generated code so that the warps
// of a block stay on the same instruction lines (the straight-line code is far larger than the
// instruction cache); the loop below is block-uniform so every thread reaches every barrier.
template <class Mech, int LM, int PREC, bool DUMP, int SYNC, int MINB>
__global__ void __launch_bounds__(kRhsMaxBlock, MINB)
    k_rhs(const double* __restrict__ sol, double* __restrict__ out, double* __restrict__ dump, long long n,
          long long ld, double p) {
  constexpr int NV = Mech::NS + 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += stride) {
    const long long i = base + threadIdx.x;
    const bool live = i < n;
    const long long ii = live ? i : n - 1;
    double s[NV], r[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = __ldcs(sol + v * ld + ii);
    if constexpr (PREC == 0)
      Mech::template rhs_fp64<LM, DUMP, SYNC>(s, p, r, DUMP && live ? dump + i : nullptr, ld);
    else
      Mech::template rhs_mixed<LM, DUMP, SYNC>(s, p, r, DUMP && live ? dump + i : nullptr, ld);
    if (live) {
#pragma unroll
      for (int v = 0; v < NV; ++v) __stcs(out + v * ld + i, r[v]);
    }
  }
}

// Launch geometry for the grid-stride rate kernel: one thread per cell up to a cap of
// 64 resident blocks' worth per SM (the loop covers the rest).
inline unsigned rhs_grid(long long n, int block) {
  long long b = (n + block - 1) / block;
  long long cap = 148LL * 64;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

// Per-cell mixture properties (csrc/props_kernels.cuh): which outputs, and where.
enum { TNG_PROPS_DENSITY = 1, TNG_PROPS_VISC = 2, TNG_PROPS_DIFF = 4 };
struct PropsArgs {
  const double* y;         // species k of cell c at y[k*ldy + c]
  long long ldy;
  const double* T;         // temperature of cell c
  const int* mask;         // mask(i,j) of the padded block (nxo x nyo), nullable
  long long nxo, nyo;
  long long n;             // cells
  double p;                // thermodynamic pressure (density)
  double *rho, *wmix;      // density outputs, nullable
  double* visc;            // viscosity output
  double* diff;            // species diffusivities, species k at diff[k*ldd + c]
  long long ldd;
  double *diff_T, *diff_Z; // temperature / mixture-fraction diffusivity (diff_Z nullable)
  const double* inv_lewis; // device, NS reciprocal Lewis numbers
};

struct SolverKernels;  // bdf_kernel.cuh

struct MechOps {
  const char* name;
  int ns, nslot, nm, nelem;
  const char* const* species;
  const double* wmol[2];
  const char* const* elements;
  const double* elem;  // nelem x ns, row-major
  // rate evaluation: prec 0/1, lm 0/1; dump may be null
  cudaError_t (*rhs)(int prec, int lm, int variant, const double* sol, double* out, double* dump, long long n,
                     long long ld, double p, int block, cudaStream_t st);
  // tables of the implicit solver
  const SvLayout* sv_layout;
  const double* sv_hd[2];  // hot doubles per literal mode
  const int* sv_hi;        // hot ints
  const int* sv_ci;        // cold ints
  const SolverKernels* sk;  // the implicit solver's kernels, specialised on this mechanism: [0] FP64, [1] mixed
  // mixture properties: lm 0/1, what = TNG_PROPS_* bits (density alone, or viscosity and/or diffusivity)
  cudaError_t (*props)(int lm, int what, const PropsArgs& a, int sm_count, cudaStream_t st);
};

// Kernel variants of the rate evaluation (the autotuner's choices): 0 = plain, 1 = block
// barriers every 48 slots, 2 = barriers + a 2-blocks-per-SM register cap.
constexpr int kRhsVariants = 3;

template <class Mech, int LM, int PREC>
cudaError_t launch_rhs_v(int variant, const double* sol, double* out, double* dump, long long n, long long ld,
                         double p, int block, cudaStream_t st) {
  const unsigned grid = rhs_grid(n, block);
  if (dump) {
    k_rhs<Mech, LM, PREC, true, 0, 1><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
    return cudaGetLastError();
  }
  if (variant < 0) variant = 2;  // measured fastest on B200: barriers every 48 slots, 2 blocks per SM
  switch (variant) {
    case 1:
      k_rhs<Mech, LM, PREC, false, 1, 1><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
      break;
    case 2:
      k_rhs<Mech, LM, PREC, false, 1, 2><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
      break;
    default:
      k_rhs<Mech, LM, PREC, false, 0, 1><<<grid, block, 0, st>>>(sol, out, dump, n, ld, p);
  }
  return cudaGetLastError();
}

template <class Mech>
cudaError_t launch_rhs(int prec, int lm, int variant, const double* sol, double* out, double* dump, long long n,
                       long long ld, double p, int block, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (block <= 0 || block > kRhsMaxBlock) block = 128;
  if (dump && lm != 0) return cudaErrorInvalidValue;
  if (prec == 0)
    return lm == 0 ? launch_rhs_v<Mech, 0, 0>(variant, sol, out, dump, n, ld, p, block, st)
                   : launch_rhs_v<Mech, 1, 0>(0, sol, out, nullptr, n, ld, p, block, st);
  return lm == 0 ? launch_rhs_v<Mech, 0, 1>(variant, sol, out, dump, n, ld, p, block, st)
                 : launch_rhs_v<Mech, 1, 1>(0, sol, out, nullptr, n, ld, p, block, st);
}

}  // namespace tng
