// The drop-in for finitechem_source_chemistry(RHO_, SC_) (combustion/finitechem.f90:962-1071):
// the solver's own Fortran arrays (column-major, with ghost layers) in, the same arrays updated.
//
// Per interior cell with mask(i,j) /= 1 (finitechem.f90:993-1065):
//   sol(1:N) = max(RHO*SC(isc_sc:isc_sc+N-1), 0),  sol(N+1) = RHO*SC(isc_T)      (:1002-1003)
//   integrate over dt                                                            (:1034)
//   SC(species) = sol(1:N)/RHO, SC(isc_T) = sol(N+1)/RHO                         (:1041-1042)
//   HR = Cp_mix(new Y, new T) * (sol(N+1) - solold(N+1)) / dt                     (:1047-1050)
//   chemsrc(1..3) = (sol - solold)/dt of H2O, CO, CO2 (skipped for absent species) (:1051-1057)
// Masked cells get dt = 0 in the compact batch (the solver leaves them untouched).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

struct FortranView {
  int imino, jmino, kmino, nxo, nyo, nzo;
  int imin, jmin, kmin, nx, ny, nz;
  long long vol;  // nxo*nyo*nzo
};

__device__ __forceinline__ long long fidx(const FortranView& v, int i, int j, int k) {
  return (long long)(i - v.imino) + (long long)v.nxo * ((j - v.jmino) + (long long)v.nyo * (k - v.kmino));
}

// interior cell c -> (i, j, k), i fastest (the reference's k, j, i loop order)
__device__ __forceinline__ void cell_ijk(const FortranView& v, long long c, int* i, int* j, int* k) {
  *i = v.imin + (int)(c % v.nx);
  const long long r = c / v.nx;
  *j = v.jmin + (int)(r % v.ny);
  *k = v.kmin + (int)(r / v.ny);
}

__global__ void k_fortran_gather(FortranView v, const double* __restrict__ rho, const double* __restrict__ spec,
                                 const double* __restrict__ temp, const int* __restrict__ mask, int ns, double dt,
                                 double* __restrict__ state, double* __restrict__ old_state, double* __restrict__ dts,
                                 long long n) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    cell_ijk(v, c, &i, &j, &k);
    const long long o = fidx(v, i, j, k);
    const bool active = !mask || mask[(long long)(i - v.imino) + (long long)v.nxo * (j - v.jmino)] != 1;
    const double r = rho[o];
    for (int s = 0; s < ns; ++s) {
      const double val = fmax(r * spec[(long long)s * v.vol + o], 0.0);
      state[(long long)s * n + c] = val;
      old_state[(long long)s * n + c] = val;
    }
    const double rt = r * temp[o];
    state[(long long)ns * n + c] = rt;
    old_state[(long long)ns * n + c] = rt;
    dts[c] = active ? dt : 0.0;
  }
}

__global__ void k_fortran_scatter(FortranView v, const double* __restrict__ rho, double* __restrict__ spec,
                                  double* __restrict__ temp, const int* __restrict__ mask, int ns,
                                  const double* __restrict__ state, const double* __restrict__ old_state, long long n,
                                  double dt, const double* __restrict__ th, double tmid, double* __restrict__ hr,
                                  double* __restrict__ chemsrc, int s_h2o, int s_co, int s_co2) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    cell_ijk(v, c, &i, &j, &k);
    const long long o = fidx(v, i, j, k);
    if (mask && mask[(long long)(i - v.imino) + (long long)v.nxo * (j - v.jmino)] == 1) continue;
    const double r = rho[o];
    double cpm = 0.0;
    const double Tn = state[(long long)ns * n + c] / r;
    const int toff = Tn > tmid ? 0 : 12;
    for (int s = 0; s < ns; ++s) {
      const double y = state[(long long)s * n + c] / r;
      spec[(long long)s * v.vol + o] = y;
      const double* a = th + kThStride * s + toff;
      cpm += y * (a[0] * (a[7] + Tn * (a[8] + Tn * (a[9] + Tn * (a[10] + Tn * a[11])))));
    }
    temp[o] = Tn;
    if (hr) hr[o] = cpm * (state[(long long)ns * n + c] - old_state[(long long)ns * n + c]) / dt;
    if (chemsrc) {
      const int sp[3] = {s_h2o, s_co, s_co2};
      for (int q = 0; q < 3; ++q)
        if (sp[q] >= 0)
          chemsrc[(long long)q * v.vol + o] = (state[(long long)sp[q] * n + c] - old_state[(long long)sp[q] * n + c]) / dt;
    }
  }
}

}  // namespace tng

namespace tng {

// The host-side checks and index arithmetic of a rank's padded block (no device involved).
static int extent_view(const tng_extent* ext, int ns, FortranView* out, int* sp3, long long* n_out) {
  if (!ext) return set_error(TNG_ERR_ARG, "tng_chem_substep: null extent");
  const tng_extent& e = *ext;
  FortranView v;
  v.imino = e.imino, v.jmino = e.jmino, v.kmino = e.kmino;
  v.nxo = e.imaxo - e.imino + 1, v.nyo = e.jmaxo - e.jmino + 1, v.nzo = e.kmaxo - e.kmino + 1;
  v.imin = e.imin, v.jmin = e.jmin, v.kmin = e.kmin;
  v.nx = e.imax - e.imin + 1, v.ny = e.jmax - e.jmin + 1, v.nz = e.kmax - e.kmin + 1;
  if (v.nxo <= 0 || v.nyo <= 0 || v.nzo <= 0 || v.nx <= 0 || v.ny <= 0 || v.nz <= 0 || e.imin < e.imino ||
      e.imax > e.imaxo || e.jmin < e.jmino || e.jmax > e.jmaxo || e.kmin < e.kmino || e.kmax > e.kmaxo)
    return set_error(TNG_ERR_ARG, "tng_chem_substep: inconsistent extents");
  if (e.isc_sc < 1 || e.isc_sc + ns - 1 > e.nscalar || e.isc_T < 1 || e.isc_T > e.nscalar ||
      (e.isc_T >= e.isc_sc && e.isc_T < e.isc_sc + ns))
    return set_error(TNG_ERR_ARG, "tng_chem_substep: scalar indices out of range");
  auto sp_index = [&](int isc) { return (isc >= e.isc_sc && isc < e.isc_sc + ns) ? isc - e.isc_sc : -1; };
  sp3[0] = sp_index(e.isc_H2O), sp3[1] = sp_index(e.isc_CO), sp3[2] = sp_index(e.isc_CO2);
  v.vol = (long long)v.nxo * v.nyo * v.nzo;
  const long long n = (long long)v.nx * v.ny * v.nz;
  if (n > 0x7fffffffLL) return set_error(TNG_ERR_ARG, "tng_chem_substep: at most 2^31-1 interior cells");
  *out = v;
  *n_out = n;
  return TNG_OK;
}

}  // namespace tng

using namespace tng;

extern "C" int tng_extent_plan(const tng_extent* ext, int nspecies, int64_t* n_interior, int64_t* volume,
                               int* diag_species) {
  if (nspecies < 1) return set_error(TNG_ERR_ARG, "tng_extent_plan: nspecies must be positive");
  FortranView v;
  int sp3[3];
  long long n = 0;
  const int rc = extent_view(ext, nspecies, &v, sp3, &n);
  if (rc) return rc;
  if (n_interior) *n_interior = n;
  if (volume) *volume = v.vol;
  if (diag_species) std::memcpy(diag_species, sp3, sizeof(sp3));
  return TNG_OK;
}

extern "C" int tng_chem_substep(tng_chem* h, const double* rho, double* sc, const int* mask, const tng_extent* ext,
                                double dt, double p_mid, double* hr, double* chemsrc, int flags,
                                tng_substep_stats* stats) {
  if (!h || !rho || !sc || !ext) return set_error(TNG_ERR_ARG, "tng_chem_substep: null argument");
  if (flags != TNG_DEVICE_PTRS && flags != TNG_HOST_PTRS) return set_error(TNG_ERR_ARG, "tng_chem_substep: bad flags");
  const tng_extent& e = *ext;
  const int ns = h->ops->ns;
  FortranView v;
  int sp3[3];
  long long n = 0;
  int rc = extent_view(ext, ns, &v, sp3, &n);
  if (rc) return rc;
  if (!(dt > 0.0) || !(p_mid > 0.0)) return set_error(TNG_ERR_ARG, "tng_chem_substep: dt and pressure must be positive");
  const int s_h2o = sp3[0], s_co = sp3[1], s_co2 = sp3[2];
  DeviceGuard g(h->cfg.device);
  rc = solver_prepare(h);
  if (rc) return rc;
  cudaStream_t st = h->stream;
  const int nv = ns + 1;
  // device views of the Fortran arrays (copies for host pointers: species block, T, rho, mask)
  const double* drho = rho;
  double* dspec = sc + (long long)(e.isc_sc - 1) * v.vol;
  double* dtemp = sc + (long long)(e.isc_T - 1) * v.vol;
  const int* dmask = mask;
  double *dhr = hr, *dcs = chemsrc;
  const size_t mask_n = (size_t)v.nxo * v.nyo;
  size_t need = (size_t)v.vol * (nv + 1 + 1 + 3) * sizeof(double) + mask_n * sizeof(int) + 256;
  if (flags == TNG_HOST_PTRS) {
    if (!h->bufs[6].reserve(need)) return set_error(TNG_ERR_CUDA, "tng_chem_substep: staging allocation failed");
    double* base = (double*)h->bufs[6].ptr;
    double* r_ = base;
    double* s_ = r_ + v.vol;
    double* t_ = s_ + (size_t)ns * v.vol;
    double* hr_ = t_ + v.vol;
    double* cs_ = hr_ + v.vol;
    int* m_ = (int*)(cs_ + 3 * v.vol);
    cudaMemcpyAsync(r_, rho, sizeof(double) * v.vol, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s_, dspec, sizeof(double) * ns * v.vol, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(t_, dtemp, sizeof(double) * v.vol, cudaMemcpyHostToDevice, st);
    if (mask) cudaMemcpyAsync(m_, mask, sizeof(int) * mask_n, cudaMemcpyHostToDevice, st);
    if (chemsrc) cudaMemcpyAsync(cs_, chemsrc, sizeof(double) * 3 * v.vol, cudaMemcpyHostToDevice, st);
    if (hr) cudaMemcpyAsync(hr_, hr, sizeof(double) * v.vol, cudaMemcpyHostToDevice, st);
    drho = r_, dspec = s_, dtemp = t_, dmask = mask ? m_ : nullptr, dhr = hr ? hr_ : nullptr;
    dcs = chemsrc ? cs_ : nullptr;
  }
  // compact batch: state, old state, per-cell dt
  if (!h->bufs[7].reserve((size_t)n * (2 * nv + 1) * sizeof(double)))
    return set_error(TNG_ERR_CUDA, "tng_chem_substep: batch allocation failed");
  double* state = (double*)h->bufs[7].ptr;
  double* old_state = state + (size_t)nv * n;
  double* dts = old_state + (size_t)nv * n;
  const int grid = (int)std::min<long long>(4096, (n + 255) / 256);
  k_fortran_gather<<<grid, 256, 0, st>>>(v, drho, dspec, dtemp, dmask, ns, dt, state, old_state, dts, n);
  rc = substep_run(h, state, n, n, dts, 0.0, p_mid, TNG_DEVICE_PTRS, nullptr, nullptr, nullptr, nullptr, nullptr, stats);
  if (rc) return rc;
  const double* th;
  double tmid;
  solver_thermo(h, &th, &tmid);
  k_fortran_scatter<<<grid, 256, 0, st>>>(v, drho, dspec, dtemp, dmask, ns, state, old_state, n, dt, th, tmid, dhr, dcs,
                                          s_h2o, s_co, s_co2);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_error(ce, "tng_chem_substep");
  if (flags == TNG_HOST_PTRS) {
    cudaMemcpyAsync(sc + (long long)(e.isc_sc - 1) * v.vol, dspec, sizeof(double) * ns * v.vol, cudaMemcpyDeviceToHost,
                    st);
    cudaMemcpyAsync(sc + (long long)(e.isc_T - 1) * v.vol, dtemp, sizeof(double) * v.vol, cudaMemcpyDeviceToHost, st);
    if (hr) cudaMemcpyAsync(hr, dhr, sizeof(double) * v.vol, cudaMemcpyDeviceToHost, st);
    if (chemsrc) cudaMemcpyAsync(chemsrc, dcs, sizeof(double) * 3 * v.vol, cudaMemcpyDeviceToHost, st);
    if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(ce, "tng_chem_substep");
  }
  return TNG_OK;
}
