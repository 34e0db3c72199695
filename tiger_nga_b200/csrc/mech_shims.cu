// Compatibility shims with the reference mechanism's Fortran signatures, for a caller that still
// evaluates the mechanism one cell at a time the way finitechem_compute_rhs does
// (combustion/finitechem.f90:93-175):
//   PRODRATES(CDOT, W, K, C, M, TEMP, PRESSURE)   e.g. combustion/HYDROGENF.f90:4-277
//   COMPTHERMODATA(H, CP, T)                      e.g. combustion/HYDROGENF.f90:514-673
// Arguments by reference (a Fortran caller writes `call tng_prodrates(...)`). They run on the GPU
// of the handle registered with tng_set_mechanism_handle -- one launch and two copies per call:
// correct, but the batch entry points are the fast path. Fortran subroutines return no status:
// on an error the outputs are set to NaN (when the sizes are known) and tng_last_error has the
// message.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <vector>

#include "tiger_chem.h"
#include "tng_runtime.h"

using namespace tng;

namespace {

std::atomic<tng_chem*> g_handle{nullptr};

__global__ void k_thermo_one(const double* __restrict__ th, double tmid, int ns, double T, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const double* a = th + kThStride * k + (T > tmid ? 0 : 12);  // T > 1000 strict, as COMPTHERMODATA
  out[k] = a[0] * (T * (a[1] + T * (a[2] + T * (a[3] + T * (a[4] + T * a[5])))) + a[6]);
  out[ns + k] = a[0] * (a[7] + T * (a[8] + T * (a[9] + T * (a[10] + T * a[11]))));
}

void fill_nan(double* p, int n) {
  for (int i = 0; p && i < n; ++i) p[i] = std::nan("");
}

}  // namespace

extern "C" void tng_set_mechanism_handle(tng_chem* h) { g_handle.store(h); }

extern "C" void tng_prodrates_(double* cdot, double* w, double* k, const double* c, double* m, const double* temp,
                               const double* pressure) {
  (void)k, (void)m;  // the reference's work arrays of rate constants and third-body sums
  tng_chem* h = g_handle.load();
  if (!h || !cdot || !c || !temp || !pressure) {
    set_error(TNG_ERR_ARG, "tng_prodrates_: no handle registered or null argument");
    return;
  }
  const int ns = h->ops->ns, nv = ns + 1, nslot = h->ops->nslot;
  const bool rates = w && h->cfg.literal_mode == TNG_LIT_REF;  // the slot rates come from the dump kernel
  DeviceGuard g(h->cfg.device);
  // the one-cell state (rho Y_k = C_k W_k, rho T) in the library's layout
  const double* W = h->ops->wmol[h->cfg.literal_mode];
  std::vector<double> hs(2 * nv + nslot);
  double rho = 0.0;
  for (int s = 0; s < ns; ++s) hs[s] = c[s] * W[s], rho += hs[s];
  hs[ns] = rho * *temp;
  if (!h->bufs[10].reserve(sizeof(double) * hs.size())) {
    set_error(TNG_ERR_CUDA, "tng_prodrates_: allocation failed");
    fill_nan(cdot, ns);
    return;
  }
  double* d = (double*)h->bufs[10].ptr;
  cudaStream_t st = h->stream;
  cudaMemcpyAsync(d, hs.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st);
  cudaError_t e = rates ? h->ops->rhs(h->cfg.precision, 0, 0, d, d + nv, d + 2 * nv, 1, 1, *pressure, 0, st)
                        : h->ops->rhs(h->cfg.precision, h->cfg.literal_mode, h->cfg.rate_variant, d, d + nv, nullptr, 1, 1,
                                      *pressure, 0, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data() + nv, d + nv, sizeof(double) * (nv + (rates ? nslot : 0)),
                                            cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cuda_error(e, "tng_prodrates_");
    fill_nan(cdot, ns);
    if (w) fill_nan(w, nslot);
    return;
  }
  for (int s = 0; s < ns; ++s) cdot[s] = hs[nv + s] / W[s];  // d(rho Y_k)/dt = CDOT_k W_k
  if (rates)
    for (int r = 0; r < nslot; ++r) w[r] = hs[2 * nv + r];
}

extern "C" void tng_compthermodata_(double* hk, double* cp, const double* t) {
  tng_chem* h = g_handle.load();
  if (!h || !hk || !cp || !t) {
    set_error(TNG_ERR_ARG, "tng_compthermodata_: no handle registered or null argument");
    return;
  }
  const int ns = h->ops->ns;
  DeviceGuard g(h->cfg.device);
  int rc = solver_prepare(h);  // the NASA tables on the device
  cudaError_t e = cudaSuccess;
  if (!rc && !h->bufs[10].reserve(sizeof(double) * 2 * ns)) rc = set_error(TNG_ERR_CUDA, "tng_compthermodata_: allocation");
  if (!rc) {
    const double* th;
    double tmid;
    solver_thermo(h, &th, &tmid);
    double* d = (double*)h->bufs[10].ptr;
    k_thermo_one<<<1, 64, 0, h->stream>>>(th, tmid, ns, *t, d);
    std::vector<double> out(2 * ns);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), d, sizeof(double) * 2 * ns, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) {
      for (int s = 0; s < ns; ++s) hk[s] = out[s], cp[s] = out[ns + s];
      return;
    }
    cuda_error(e, "tng_compthermodata_");
  }
  fill_nan(hk, ns);
  fill_nan(cp, ns);
}
