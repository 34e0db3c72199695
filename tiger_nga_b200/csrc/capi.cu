// C-ABI implementation (include/tiger_chem.h): handles, streams, staging and dispatch to the
// per-mechanism kernels. Host runtime in C++; every compute call runs on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_error(cudaError_t e, const char* what) {
  return set_error(TNG_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

const MechOps* find_mech(const char* name) {
  const MechOps* const* all = all_mechanisms();
  for (int i = 0; all[i]; ++i)
    if (std::strcmp(all[i]->name, name) == 0) return all[i];
  return nullptr;
}

}  // namespace tng

using namespace tng;

extern "C" {

void tng_default_cfg(tng_cfg* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->precision = TNG_FP64;
  cfg->literal_mode = TNG_LIT_REF;
  cfg->device = 0;
  cfg->rtol = 1.0e-6;
  cfg->atol = 1.0e-12;
  cfg->max_steps = 10000;
  cfg->max_newton = 4;
  cfg->block_size = 0;
  cfg->rate_variant = -1;
  cfg->solver_warps = 0;
  cfg->pass_budget = 0;
  cfg->max_passes = 8;
}

int tng_last_error(char* buf, int len) {
  int n = (int)g_last_error.size();
  if (buf && len > 0) {
    int c = std::min(n, len - 1);
    std::memcpy(buf, g_last_error.data(), c);
    buf[c] = 0;
  }
  return n;
}

int tng_chem_create(const char* mechanism, const tng_cfg* cfg, tng_chem** out) {
  if (!mechanism || !out) return set_error(TNG_ERR_ARG, "tng_chem_create: null argument");
  *out = nullptr;
  const MechOps* ops = find_mech(mechanism);
  if (!ops) return set_error(TNG_ERR_MECH, "tng_chem_create: unknown mechanism '%s'", mechanism);
  tng_cfg c;
  if (cfg)
    c = *cfg;
  else
    tng_default_cfg(&c);
  if (c.precision != TNG_FP64 && c.precision != TNG_MIXED)
    return set_error(TNG_ERR_ARG, "tng_chem_create: precision must be TNG_FP64 or TNG_MIXED");
  if (c.literal_mode != TNG_LIT_REF && c.literal_mode != TNG_LIT_F64)
    return set_error(TNG_ERR_ARG, "tng_chem_create: literal_mode must be TNG_LIT_REF or TNG_LIT_F64");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return set_error(TNG_ERR_CUDA, "tng_chem_create: no CUDA device (%s); this library has no CPU path",
                     cudaGetErrorString(e));
  if (c.device < 0 || c.device >= ndev) return set_error(TNG_ERR_ARG, "tng_chem_create: bad device %d", c.device);
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, c.device)) != cudaSuccess) return cuda_error(e, "cudaGetDeviceProperties");
  if (prop.major != 10)
    return set_error(TNG_ERR_CUDA, "tng_chem_create: device %d is sm_%d%d; this build targets sm_100a", c.device,
                     prop.major, prop.minor);
  tng_chem* h = new tng_chem();
  h->ops = ops;
  h->cfg = c;
  h->sm_count = prop.multiProcessorCount;
  DeviceGuard g(c.device);
  if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete h;
    return cuda_error(e, "cudaStreamCreate");
  }
  for (int i = 0; i < 2; ++i) {
    if ((e = cudaStreamCreateWithFlags(&h->copy_stream[i], cudaStreamNonBlocking)) != cudaSuccess) {
      tng_chem_destroy(h);
      return cuda_error(e, "cudaStreamCreate");
    }
  }
  *out = h;
  return TNG_OK;
}

int tng_chem_destroy(tng_chem* h) {
  if (!h) return TNG_OK;
  if (h->dependents > 0)
    return set_error(TNG_ERR_STATE, "tng_chem_destroy: %d network/surrogate objects still use this handle",
                     h->dependents);
  {
    DeviceGuard g(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    solver_release(h);
    for (auto& b : h->bufs) b.release();
    for (int i = 0; i < 2; ++i)
      if (h->copy_stream[i]) cudaStreamDestroy(h->copy_stream[i]);
    if (h->stream) cudaStreamDestroy(h->stream);
  }
  delete h;
  return TNG_OK;
}

int tng_chem_sizes(const tng_chem* h, int* ns, int* nslot, int* nm) {
  if (!h) return set_error(TNG_ERR_ARG, "tng_chem_sizes: null handle");
  if (ns) *ns = h->ops->ns;
  if (nslot) *nslot = h->ops->nslot;
  if (nm) *nm = h->ops->nm;
  return TNG_OK;
}

int tng_chem_molar_mass(const tng_chem* h, double* wmol) {
  if (!h || !wmol) return set_error(TNG_ERR_ARG, "tng_chem_molar_mass: null argument");
  std::memcpy(wmol, h->ops->wmol[h->cfg.literal_mode], sizeof(double) * h->ops->ns);
  return TNG_OK;
}

int tng_chem_species_name(const tng_chem* h, int k, char* buf, int len) {
  if (!h || !buf || len <= 0) return set_error(TNG_ERR_ARG, "tng_chem_species_name: bad argument");
  if (k < 0 || k >= h->ops->ns) return set_error(TNG_ERR_ARG, "tng_chem_species_name: species %d out of range", k);
  std::snprintf(buf, len, "%s", h->ops->species[k]);
  return TNG_OK;
}

void* tng_chem_stream(tng_chem* h) { return h ? (void*)h->stream : nullptr; }

int tng_chem_sync(tng_chem* h) {
  if (!h) return set_error(TNG_ERR_ARG, "tng_chem_sync: null handle");
  DeviceGuard g(h->cfg.device);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_error(e, "tng_chem_sync");
  return TNG_OK;
}

int tng_prodrates_batch(tng_chem* h, const double* sol, double* rhs, int64_t ncells, int64_t ld, double p,
                        int flags) {
  if (!h) return set_error(TNG_ERR_ARG, "tng_prodrates_batch: null handle");
  if (ncells < 0 || ld < ncells) return set_error(TNG_ERR_ARG, "tng_prodrates_batch: need 0 <= ncells <= ld");
  if (ncells == 0) return TNG_OK;
  if (!sol || !rhs) return set_error(TNG_ERR_ARG, "tng_prodrates_batch: null array");
  if (!(p > 0.0)) return set_error(TNG_ERR_ARG, "tng_prodrates_batch: pressure must be positive");
  DeviceGuard g(h->cfg.device);
  const int nv = h->ops->ns + 1;
  const int prec = h->cfg.precision, lm = h->cfg.literal_mode, blk = h->cfg.block_size;
  cudaError_t e;
  if (flags == TNG_DEVICE_PTRS) {
    e = h->ops->rhs(prec, lm, h->cfg.rate_variant, sol, rhs, nullptr, ncells, ld, p, blk, h->stream);
    if (e != cudaSuccess) return cuda_error(e, "rate kernel launch");
    return TNG_OK;
  }
  if (flags != TNG_HOST_PTRS) return set_error(TNG_ERR_ARG, "tng_prodrates_batch: bad flags %d", flags);
  // Host arrays: pipeline chunks through two device buffer pairs so the host->device copy of
  // chunk c+1, the kernel on chunk c and the device->host copy of chunk c-1 overlap.
  const int64_t chunk = std::min<int64_t>(ncells, 1 << 18);
  const size_t bytes = (size_t)nv * chunk * sizeof(double);
  for (int i = 0; i < 4; ++i)
    if (!h->bufs[i].reserve(bytes)) return set_error(TNG_ERR_CUDA, "device buffer allocation of %zu bytes failed", bytes);
  cudaEvent_t ev_in[2], ev_k[2];
  for (int i = 0; i < 2; ++i) {
    cudaEventCreateWithFlags(&ev_in[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_k[i], cudaEventDisableTiming);
  }
  int rc = TNG_OK;
  int nchunk = (int)((ncells + chunk - 1) / chunk);
  for (int c = 0; c < nchunk && rc == TNG_OK; ++c) {
    const int b = c & 1;
    const int64_t i0 = (int64_t)c * chunk;
    const int64_t n = std::min<int64_t>(chunk, ncells - i0);
    double* din = (double*)h->bufs[b].ptr;
    double* dout = (double*)h->bufs[2 + b].ptr;
    cudaStream_t cs = h->copy_stream[b];
    // the buffers of slot b are free once the previous kernel on them is done and its output copied
    if ((e = cudaMemcpy2DAsync(din, n * sizeof(double), sol + i0, ld * sizeof(double), n * sizeof(double), nv,
                               cudaMemcpyHostToDevice, cs)) != cudaSuccess) {
      rc = cuda_error(e, "host->device copy");
      break;
    }
    cudaEventRecord(ev_in[b], cs);
    cudaStreamWaitEvent(h->stream, ev_in[b], 0);
    if ((e = h->ops->rhs(prec, lm, h->cfg.rate_variant, din, dout, nullptr, n, n, p, blk, h->stream)) != cudaSuccess) {
      rc = cuda_error(e, "rate kernel launch");
      break;
    }
    cudaEventRecord(ev_k[b], h->stream);
    cudaStreamWaitEvent(cs, ev_k[b], 0);
    if ((e = cudaMemcpy2DAsync(rhs + i0, ld * sizeof(double), dout, n * sizeof(double), n * sizeof(double), nv,
                               cudaMemcpyDeviceToHost, cs)) != cudaSuccess) {
      rc = cuda_error(e, "device->host copy");
      break;
    }
  }
  for (int i = 0; i < 2; ++i) {
    if ((e = cudaStreamSynchronize(h->copy_stream[i])) != cudaSuccess && rc == TNG_OK) rc = cuda_error(e, "copy stream");
    cudaEventDestroy(ev_in[i]);
    cudaEventDestroy(ev_k[i]);
  }
  if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess && rc == TNG_OK) rc = cuda_error(e, "rate kernel");
  return rc;
}

int tng_prodrates_batch_rates(tng_chem* h, const double* sol, double* rhs, double* rates, int64_t ncells, int64_t ld,
                              double p) {
  if (!h || !sol || !rhs || !rates) return set_error(TNG_ERR_ARG, "tng_prodrates_batch_rates: null argument");
  if (ncells < 0 || ld < ncells) return set_error(TNG_ERR_ARG, "tng_prodrates_batch_rates: need 0 <= ncells <= ld");
  if (h->cfg.literal_mode != TNG_LIT_REF)
    return set_error(TNG_ERR_ARG, "tng_prodrates_batch_rates: only built for TNG_LIT_REF");
  DeviceGuard g(h->cfg.device);
  cudaError_t e = h->ops->rhs(h->cfg.precision, 0, 0, sol, rhs, rates, ncells, ld, p, h->cfg.block_size, h->stream);
  if (e != cudaSuccess) return cuda_error(e, "rate kernel launch");
  return TNG_OK;
}

}  // extern "C"
