// Mixture-property kernels around the substep (sm_100a): finitechem_W + finitechem_density
// (combustion/finitechem.f90:65-74, :324-345), finitechem_viscosity (:351-406) and
// finitechem_diffusivity (:412-461) with finitechem_omegamu (:467-487).
//
// One cell per thread over the cells of a species-major array (species k of cell c at
// y[k*ldy + c]; the reference's SC(i,j,k,isc_sc+k-1) block with the padded volume as ld), so
// every load and store of a warp is one contiguous segment. The per-cell arithmetic is the
// mechanism's generated code (Mech::mix_w, Mech::transport). The viscosity keeps
// three per-cell vectors of NS doubles in shared memory (one slice per thread, stride
// kPropsBlock; the first vector stages the mass fractions), which bounds residency at
// (smem per SM) / (32 NS bytes) threads.
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace tng {

constexpr int kPropsBlock = 64;

// shared memory of a transport block: per thread 3 vectors of NS doubles with the viscosity
// (the first one stages the mass fractions), NS doubles for the diffusivities alone
template <class Mech>
constexpr int props_smem(int what) {
  return ((what & TNG_PROPS_VISC) ? 3 : 1) * Mech::NS * kPropsBlock * (int)sizeof(double);
}

// Viscosity and / or diffusivities (WHAT = TNG_PROPS_VISC / TNG_PROPS_DIFF bits).
template <class Mech, int LM, int WHAT>
__global__ void __launch_bounds__(kPropsBlock) k_props(PropsArgs a) {
  extern __shared__ double props_sv[];
  double* sv = props_sv + threadIdx.x;
  const long long stride = (long long)gridDim.x * kPropsBlock;
  for (long long c = (long long)blockIdx.x * kPropsBlock + threadIdx.x; c < a.n; c += stride) {
    if (a.mask) {
      const long long i = c % a.nxo;
      const long long j = (c / a.nxo) % a.nyo;
      if (__ldg(a.mask + i + (long long)a.nxo * j) == 1) continue;
    }
    const double T = __ldcs(a.T + c);
    double visc = 0.0, lc = 0.0;
    Mech::template transport<LM, (WHAT & TNG_PROPS_VISC) != 0, (WHAT & TNG_PROPS_DIFF) != 0, kPropsBlock>(
        a.y + c, a.ldy, T, sv, &visc, &lc);
    if constexpr ((WHAT & TNG_PROPS_VISC) != 0) __stcs(a.visc + c, visc);
    if constexpr ((WHAT & TNG_PROPS_DIFF) != 0) {
      // DIFF(species k) = (lambda/Cp_mix)/Lewis_k, DIFF(T) = DIFF(ZMIX) = lambda/Cp_mix (:444-451)
#pragma unroll 4
      for (int k = 0; k < Mech::NS; ++k) __stcs(a.diff + k * a.ldd + c, lc * __ldg(a.inv_lewis + k));
      __stcs(a.diff_T + c, lc);
      if (a.diff_Z) __stcs(a.diff_Z + c, lc);
    }
  }
}

// Density and W_mix: a streaming kernel (N+1 loads, two stores per cell).
constexpr int kDensityBlock = 256;
template <class Mech, int LM>
__global__ void __launch_bounds__(kDensityBlock) k_density(PropsArgs a) {
  const long long stride = (long long)gridDim.x * kDensityBlock;
  for (long long c = (long long)blockIdx.x * kDensityBlock + threadIdx.x; c < a.n; c += stride) {
    if (a.mask) {
      const long long i = c % a.nxo;
      const long long j = (c / a.nxo) % a.nyo;
      if (__ldg(a.mask + i + (long long)a.nxo * j) == 1) continue;
    }
    const double wm = Mech::template mix_w<LM>(a.y + c, a.ldy);
    // RHO = P_thermo * W_mix / (R_cst * T), R_cst = 8314.34 (finitechem.f90:15, :338)
    if (a.rho) __stcs(a.rho + c, a.p * wm / (8314.34 * __ldcs(a.T + c)));
    if (a.wmix) __stcs(a.wmix + c, wm);
  }
}

// Resident blocks per SM of a kernel, set up once per device (the shared-memory opt-in is a
// per-device attribute); grid = min(blocks needed, SMs x resident blocks) for the grid-stride loop.
template <class K>
cudaError_t launch_grid_stride(K kern, int block, int smem, const PropsArgs& a, int sm_count, cudaStream_t st,
                               int* occ_dev) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  int& occ = occ_dev[dev];
  if (occ == 0) {
    if (smem > 48 * 1024 && (e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
                                cudaSuccess)
      return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, block, smem);
    if (e != cudaSuccess) return e;
    occ = o < 1 ? 1 : o;
  }
  long long blocks = (a.n + block - 1) / block;
  const long long cap = (long long)sm_count * occ;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  kern<<<(unsigned)blocks, block, smem, st>>>(a);
  return cudaGetLastError();
}

template <class Mech, int LM, int WHAT>
cudaError_t launch_props_w(const PropsArgs& a, int sm_count, cudaStream_t st) {
  static int occ_dev[64] = {};
  if constexpr (WHAT == TNG_PROPS_DENSITY)
    return launch_grid_stride(k_density<Mech, LM>, kDensityBlock, 0, a, sm_count, st, occ_dev);
  else
    return launch_grid_stride(k_props<Mech, LM, WHAT>, kPropsBlock, props_smem<Mech>(WHAT), a, sm_count, st, occ_dev);
}

template <class Mech>
cudaError_t launch_props(int lm, int what, const PropsArgs& a, int sm_count, cudaStream_t st) {
#define TNG_PROPS_CASE(W)                                                                     \
  case W:                                                                                     \
    return lm ? launch_props_w<Mech, 1, W>(a, sm_count, st) : launch_props_w<Mech, 0, W>(a, sm_count, st);
  switch (what) {
    TNG_PROPS_CASE(TNG_PROPS_DENSITY)
    TNG_PROPS_CASE(TNG_PROPS_VISC)
    TNG_PROPS_CASE(TNG_PROPS_DIFF)
    TNG_PROPS_CASE(TNG_PROPS_VISC | TNG_PROPS_DIFF)
    default:
      return cudaErrorInvalidValue;
  }
#undef TNG_PROPS_CASE
}

}  // namespace tng
