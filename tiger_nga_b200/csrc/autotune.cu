// The project's autotuner: times the candidate launch configurations of the rate kernel
// (kernel variant x block size) and of the implicit solver (cells per block x pass budget, i.e.
// with or without recompaction between passes) on the caller's own cells, and keeps the fastest
// in the handle. Every candidate computes the same per-cell results (a cell's integration does not
// depend on which warp runs it, and a pass boundary saves and restores its history exactly), so
// tuning changes the speed only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

// a strided sample of m cells (and their dt) into a compact batch
__global__ void k_tune_sample(const double* __restrict__ src, long long ld, int nv, long long n, long long m,
                              const double* __restrict__ dts, double* __restrict__ dst, double* __restrict__ dts_out) {
  const long long stride = n / m;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (long long)gridDim.x * blockDim.x) {
    const long long c = j * stride;
    for (int v = 0; v < nv; ++v) dst[(long long)v * m + j] = src[(long long)v * ld + c];
    if (dts) dts_out[j] = dts[c];
  }
}

static void put(tng_tune_result* out, int a, int b, double ms) {
  if (out && out->n < TNG_TUNE_MAX) {
    out->a[out->n] = a;
    out->b[out->n] = b;
    out->ms[out->n] = ms;
    out->n++;
  }
}

}  // namespace tng

using namespace tng;

extern "C" int tng_chem_set_tuning(tng_chem* h, int rate_variant, int block_size, int solver_warps, int pass_budget) {
  if (!h) return set_error(TNG_ERR_ARG, "tng_chem_set_tuning: null handle");
  if (rate_variant < -1 || rate_variant > 2 || block_size < 0 || block_size > 1024 ||
      !(solver_warps == 0 || solver_warps == 2 || solver_warps == 4 || solver_warps == 8 || solver_warps == 16) ||
      pass_budget < 0)
    return set_error(TNG_ERR_ARG, "tng_chem_set_tuning: value out of range");
  h->cfg.rate_variant = rate_variant;
  h->cfg.block_size = block_size;
  h->cfg.solver_warps = solver_warps == 16 ? 8 : solver_warps;  // 16: 8 warps, two blocks per SM
  h->cfg.solver_occupancy = solver_warps == 16 ? 2 : 1;
  h->cfg.pass_budget = pass_budget;
  return TNG_OK;
}

extern "C" int tng_rates_autotune(tng_chem* h, const double* state, int64_t ncells, int64_t ld, double p,
                                  tng_tune_result* out) {
  if (!h || !state || ncells <= 0 || ld < ncells || !(p > 0.0))
    return set_error(TNG_ERR_ARG, "tng_rates_autotune: bad argument");
  if (out) std::memset(out, 0, sizeof(*out));
  DeviceGuard g(h->cfg.device);
  const int nv = h->ops->ns + 1;
  double* rhs = nullptr;
  cudaError_t e = cudaMalloc(&rhs, sizeof(double) * nv * ncells);
  if (e != cudaSuccess) return cuda_error(e, "tng_rates_autotune");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int variants[3] = {0, 1, 2}, blocks[3] = {64, 128, 256};
  double best = 1e300;
  int bv = -1, bb = 0;
  const tng_cfg saved = h->cfg;
  for (int v : variants)
    for (int b : blocks) {
      h->cfg.rate_variant = v;
      h->cfg.block_size = b;
      e = h->ops->rhs(h->cfg.precision, h->cfg.literal_mode, v, state, rhs, nullptr, ncells, ld, p, b, h->stream);
      if (e != cudaSuccess) break;
      cudaEventRecord(e0, h->stream);
      for (int r = 0; r < 5; ++r) h->ops->rhs(h->cfg.precision, h->cfg.literal_mode, v, state, rhs, nullptr, ncells, ld, p, b, h->stream);
      cudaEventRecord(e1, h->stream);
      if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      put(out, v, b, ms / 5.0);
      if (ms / 5.0 < best) best = ms / 5.0, bv = v, bb = b;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(rhs);
  h->cfg = saved;
  if (e != cudaSuccess) return cuda_error(e, "tng_rates_autotune");
  h->cfg.rate_variant = bv;
  h->cfg.block_size = bb;
  if (out) {
    for (int i = 0; i < out->n; ++i)
      if (out->a[i] == bv && out->b[i] == bb) out->best = i;
  }
  return TNG_OK;
}

extern "C" int tng_substep_autotune(tng_chem* h, const double* state, int64_t ncells, int64_t ld, const double* dts,
                                    double dt, double p, int64_t sample, tng_tune_result* out) {
  if (!h || !state || ncells <= 0 || ld < ncells || !(p > 0.0) || (!dts && !(dt >= 0.0)))
    return set_error(TNG_ERR_ARG, "tng_substep_autotune: bad argument");
  if (out) std::memset(out, 0, sizeof(*out));
  DeviceGuard g(h->cfg.device);
  const int nv = h->ops->ns + 1;
  const int64_t m = std::max<int64_t>(1, std::min<int64_t>(sample > 0 ? sample : 65536, ncells));
  double* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, sizeof(double) * (2 * nv * m + m));
  if (e != cudaSuccess) return cuda_error(e, "tng_substep_autotune");
  double* pristine = buf;
  double* work = buf + (size_t)nv * m;
  double* sdts = work + (size_t)nv * m;
  k_tune_sample<<<(int)std::min<int64_t>(1024, (m + 127) / 128), 128, 0, h->stream>>>(state, ld, nv, ncells, m, dts,
                                                                                       pristine, sdts);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // warps per block; 16 stands for 8 warps with launch bounds for two blocks per SM
  const int warps[4] = {2, 4, 8, 16}, budgets[3] = {0, 32, 128};
  double best = 1e300;
  int bw = 8, bb = 0;
  const tng_cfg saved = h->cfg;
  int rc = TNG_OK;
  for (int w : warps)
    for (int b : budgets) {
      h->cfg.solver_warps = w == 16 ? 8 : w;
      h->cfg.solver_occupancy = w == 16 ? 2 : 1;
      h->cfg.pass_budget = b;
      // first run builds the pass graph of this configuration; the second is timed
      for (int rep = 0; rep < 2 && !rc; ++rep) {
        cudaMemcpyAsync(work, pristine, sizeof(double) * nv * m, cudaMemcpyDeviceToDevice, h->stream);
        if (rep == 1) cudaEventRecord(e0, h->stream);
        rc = substep_run(h, work, m, m, dts ? sdts : nullptr, dt, p, TNG_DEVICE_PTRS, nullptr, nullptr, nullptr,
                         nullptr, nullptr, nullptr);
        if (rep == 1) cudaEventRecord(e1, h->stream);
      }
      if (rc) break;
      if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      put(out, w, b, ms);
      if (ms < best) best = ms, bw = w, bb = b;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(h->stream);
  cudaFree(buf);
  h->cfg = saved;
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_error(e, "tng_substep_autotune");
  h->cfg.solver_warps = bw == 16 ? 8 : bw;
  h->cfg.solver_occupancy = bw == 16 ? 2 : 1;
  h->cfg.pass_budget = bb;
  if (out) {
    for (int i = 0; i < out->n; ++i)
      if (out->a[i] == bw && out->b[i] == bb) out->best = i;
  }
  return TNG_OK;
}
