// Drop-ins for the per-cell mixture properties that surround the chemistry substep, on the
// solver's own Fortran arrays (column-major, ghost layers included):
//   tng_chem_density   <- finitechem_density + finitechem_W   (combustion/finitechem.f90:324-345, :65-74)
//   tng_chem_transport <- finitechem_viscosity + finitechem_diffusivity + finitechem_omegamu
//                                                             (finitechem.f90:351-406, :412-461, :467-487)
// The reference loops over every cell of the padded block (k = kmino_..kmaxo_, j, i) with
// mask(i,j) /= 1; the species block SC(:,:,:,isc_sc:isc_sc+N-1) is species-major with the
// padded volume as stride, which is the kernels' native layout, so the device path reads the
// arrays in place. Kernels: csrc/props_kernels.cuh over the generated per-mechanism code.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "tiger_chem.h"
#include "tng_runtime.h"

using namespace tng;

namespace {

struct Block {
  long long nxo, nyo, nzo, vol;
};

int check_extent(const tng_chem* h, const tng_extent* ext, const char* who, Block* b) {
  if (!ext) return set_error(TNG_ERR_ARG, "%s: null extent", who);
  const tng_extent& e = *ext;
  b->nxo = (long long)e.imaxo - e.imino + 1;
  b->nyo = (long long)e.jmaxo - e.jmino + 1;
  b->nzo = (long long)e.kmaxo - e.kmino + 1;
  if (b->nxo <= 0 || b->nyo <= 0 || b->nzo <= 0) return set_error(TNG_ERR_ARG, "%s: empty padded block", who);
  b->vol = b->nxo * b->nyo * b->nzo;
  const int ns = h->ops->ns;
  if (e.isc_sc < 1 || e.isc_sc + ns - 1 > e.nscalar || e.isc_T < 1 || e.isc_T > e.nscalar ||
      (e.isc_T >= e.isc_sc && e.isc_T < e.isc_sc + ns))
    return set_error(TNG_ERR_ARG, "%s: scalar indices out of range", who);
  return TNG_OK;
}

}  // namespace

extern "C" int tng_chem_density(tng_chem* h, double* rho, double* wmix, const double* sc, const int* mask,
                                const tng_extent* ext, double p_thermo, int flags) {
  if (!h || !sc) return set_error(TNG_ERR_ARG, "tng_chem_density: null argument");
  if (flags != TNG_DEVICE_PTRS && flags != TNG_HOST_PTRS) return set_error(TNG_ERR_ARG, "tng_chem_density: bad flags");
  Block b;
  int rc = check_extent(h, ext, "tng_chem_density", &b);
  if (rc) return rc;
  if (!(p_thermo > 0.0)) return set_error(TNG_ERR_ARG, "tng_chem_density: pressure must be positive");
  if (!rho && !wmix) return TNG_OK;
  DeviceGuard g(h->cfg.device);
  cudaStream_t st = h->stream;
  const int ns = h->ops->ns;
  const tng_extent& e = *ext;
  PropsArgs a{};
  a.ldy = b.vol;
  a.nxo = b.nxo, a.nyo = b.nyo, a.n = b.vol, a.p = p_thermo;
  const size_t vb = sizeof(double) * (size_t)b.vol, mb = sizeof(int) * (size_t)(b.nxo * b.nyo);
  if (flags == TNG_DEVICE_PTRS) {
    a.y = sc + (long long)(e.isc_sc - 1) * b.vol;
    a.T = sc + (long long)(e.isc_T - 1) * b.vol;
    a.mask = mask, a.rho = rho, a.wmix = wmix;
  } else {
    if (!h->bufs[9].reserve(vb * (ns + 3) + mb + 256))
      return set_error(TNG_ERR_CUDA, "tng_chem_density: staging allocation failed");
    double* y = (double*)h->bufs[9].ptr;
    double* T = y + (size_t)ns * b.vol;
    double* r = T + b.vol;
    double* w = r + b.vol;
    int* m = (int*)(w + b.vol);
    cudaMemcpyAsync(y, sc + (long long)(e.isc_sc - 1) * b.vol, vb * ns, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(T, sc + (long long)(e.isc_T - 1) * b.vol, vb, cudaMemcpyHostToDevice, st);
    if (mask) {  // masked cells keep the caller's values
      cudaMemcpyAsync(m, mask, mb, cudaMemcpyHostToDevice, st);
      if (rho) cudaMemcpyAsync(r, rho, vb, cudaMemcpyHostToDevice, st);
      if (wmix) cudaMemcpyAsync(w, wmix, vb, cudaMemcpyHostToDevice, st);
    }
    a.y = y, a.T = T, a.mask = mask ? m : nullptr, a.rho = rho ? r : nullptr, a.wmix = wmix ? w : nullptr;
  }
  cudaError_t ce = h->ops->props(h->cfg.literal_mode, TNG_PROPS_DENSITY, a, h->sm_count, st);
  if (ce != cudaSuccess) return cuda_error(ce, "tng_chem_density");
  if (flags == TNG_HOST_PTRS) {
    if (rho) cudaMemcpyAsync(rho, a.rho, vb, cudaMemcpyDeviceToHost, st);
    if (wmix) cudaMemcpyAsync(wmix, a.wmix, vb, cudaMemcpyDeviceToHost, st);
    if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(ce, "tng_chem_density");
  }
  return TNG_OK;
}

extern "C" int tng_chem_transport(tng_chem* h, double* visc, double* diff, const double* sc, const int* mask,
                                  const tng_extent* ext, const double* lewis, int isc_zmix, int flags) {
  if (!h || !sc) return set_error(TNG_ERR_ARG, "tng_chem_transport: null argument");
  if (flags != TNG_DEVICE_PTRS && flags != TNG_HOST_PTRS)
    return set_error(TNG_ERR_ARG, "tng_chem_transport: bad flags");
  Block b;
  int rc = check_extent(h, ext, "tng_chem_transport", &b);
  if (rc) return rc;
  const tng_extent& e = *ext;
  const int ns = h->ops->ns;
  if (isc_zmix < 0 || isc_zmix > e.nscalar || isc_zmix == e.isc_T ||
      (isc_zmix >= e.isc_sc && isc_zmix < e.isc_sc + ns))
    return set_error(TNG_ERR_ARG, "tng_chem_transport: isc_zmix out of range");
  if (!visc && !diff) return TNG_OK;
  std::vector<double> inv(ns, 1.0);
  if (lewis) {
    for (int k = 0; k < ns; ++k) {
      if (!(lewis[k] > 0.0)) return set_error(TNG_ERR_ARG, "tng_chem_transport: Lewis numbers must be positive");
      inv[k] = 1.0 / lewis[k];
    }
  }
  if (ns > 64) return set_error(TNG_ERR_ARG, "tng_chem_transport: more than 64 species");
  DeviceGuard g(h->cfg.device);
  cudaStream_t st = h->stream;
  // the device copy of the reciprocal Lewis numbers is refreshed only when they change (a copy
  // from pageable memory would wait for the stream, and the values rarely change between calls)
  if (h->props_lewis_n != ns || std::memcmp(h->props_inv_lewis, inv.data(), sizeof(double) * ns) != 0) {
    if (!h->bufs[8].reserve(sizeof(double) * ns))
      return set_error(TNG_ERR_CUDA, "tng_chem_transport: allocation failed");
    // stream-ordered: an earlier launch that still reads the previous values finishes first
    cudaError_t ce = cudaMemcpyAsync(h->bufs[8].ptr, inv.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return cuda_error(ce, "tng_chem_transport");
    std::memcpy(h->props_inv_lewis, inv.data(), sizeof(double) * ns);
    h->props_lewis_n = ns;
  }
  PropsArgs a{};
  a.ldy = b.vol, a.ldd = b.vol;
  a.nxo = b.nxo, a.nyo = b.nyo, a.n = b.vol;
  a.inv_lewis = (const double*)h->bufs[8].ptr;
  const size_t vb = sizeof(double) * (size_t)b.vol, mb = sizeof(int) * (size_t)(b.nxo * b.nyo);
  const long long osp = (long long)(e.isc_sc - 1) * b.vol, oT = (long long)(e.isc_T - 1) * b.vol;
  const long long oZ = (long long)(isc_zmix - 1) * b.vol;
  double *d_sp = nullptr, *d_T = nullptr, *d_Z = nullptr, *d_visc = visc;
  if (flags == TNG_DEVICE_PTRS) {
    a.y = sc + osp, a.T = sc + oT, a.mask = mask;
    if (diff) d_sp = diff + osp, d_T = diff + oT, d_Z = isc_zmix ? diff + oZ : nullptr;
  } else {
    const int nout = (visc ? 1 : 0) + (diff ? ns + 1 + (isc_zmix ? 1 : 0) : 0);
    if (!h->bufs[9].reserve(vb * (ns + 1 + nout) + mb + 256))
      return set_error(TNG_ERR_CUDA, "tng_chem_transport: staging allocation failed");
    double* y = (double*)h->bufs[9].ptr;
    double* T = y + (size_t)ns * b.vol;
    double* o = T + b.vol;
    if (visc) d_visc = o, o += b.vol;
    if (diff) {
      d_sp = o, o += (size_t)ns * b.vol;
      d_T = o, o += b.vol;
      if (isc_zmix) d_Z = o, o += b.vol;
    }
    int* m = (int*)o;
    cudaMemcpyAsync(y, sc + osp, vb * ns, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(T, sc + oT, vb, cudaMemcpyHostToDevice, st);
    if (mask) {  // masked cells keep the caller's values
      cudaMemcpyAsync(m, mask, mb, cudaMemcpyHostToDevice, st);
      if (visc) cudaMemcpyAsync(d_visc, visc, vb, cudaMemcpyHostToDevice, st);
      if (diff) {
        cudaMemcpyAsync(d_sp, diff + osp, vb * ns, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_T, diff + oT, vb, cudaMemcpyHostToDevice, st);
        if (d_Z) cudaMemcpyAsync(d_Z, diff + oZ, vb, cudaMemcpyHostToDevice, st);
      }
    }
    a.y = y, a.T = T, a.mask = mask ? m : nullptr;
  }
  a.visc = d_visc, a.diff = d_sp, a.diff_T = d_T, a.diff_Z = d_Z;
  const int what = (visc ? TNG_PROPS_VISC : 0) | (diff ? TNG_PROPS_DIFF : 0);
  cudaError_t ce = h->ops->props(h->cfg.literal_mode, what, a, h->sm_count, st);
  if (ce != cudaSuccess) return cuda_error(ce, "tng_chem_transport");
  if (flags == TNG_HOST_PTRS) {
    if (visc) cudaMemcpyAsync(visc, d_visc, vb, cudaMemcpyDeviceToHost, st);
    if (diff) {
      cudaMemcpyAsync(diff + osp, d_sp, vb * ns, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(diff + oT, d_T, vb, cudaMemcpyDeviceToHost, st);
      if (d_Z) cudaMemcpyAsync(diff + oZ, d_Z, vb, cudaMemcpyDeviceToHost, st);
    }
    if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(ce, "tng_chem_transport");
  }
  return TNG_OK;
}
