// Host side of the implicit substep: solver tables on the device, scratch, the pass loop as a
// CUDA graph, statistics, and the C-ABI entry points tng_substep_batch / tng_solver_rhs_jac.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "bdf_kernel.cuh"
#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

// The BDF coefficients: l(x) = prod_{i=1..q} (1 + x/i) normalised to l_1 = 1, and the error
// constants of orders q, q-1 and q+1 (same arithmetic as oracle/solver_oracle.c).
BdfCoef make_coef() {
  BdfCoef c;
  std::memset(&c, 0, sizeof(c));
  for (int q = 1; q <= kQmax + 1; ++q) {
    double v[kQmax + 3] = {1.0};
    for (int i = 1; i <= q; ++i)
      for (int j = i; j >= 1; --j) v[j] += v[j - 1] / (double)i;
    for (int j = 0; j <= q; ++j) c.L[q][j] = v[j] / v[1];
  }
  double fact = 1.0;
  for (int q = 1; q <= kQmax; ++q) {
    fact *= q;
    c.errc[q] = c.L[q][0] / (q + 1) * fact * c.L[q][q];
    c.dnc[q] = q > 1 ? c.L[q - 1][0] / q * fact : 0.0;
    c.upc[q] = c.L[q + 1][0] / (q + 2) * fact * c.L[q][q];
  }
  for (int e = 1; e <= kQmax + 2; ++e) c.grow[e] = std::pow(2.0 / 3.0, e) * (1.0 + 1e-9);
  return c;
}

struct SubstepKey {
  const double* state;
  int64_t ncells, ld;
  const int* list;
  const int* nlist;
  const double* dts;
  double dt, p;
  int warps, occ, budget, passes;
  int* nst;
  int* nni;
  int* status;
  bool operator==(const SubstepKey& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

struct SolverState {
  bool tables_ready = false;
  SvDev dev{};
  BdfCoef* d_coef = nullptr;  // BDF coefficients on the device (staged into shared memory by the kernel)
  int* d_int = nullptr;  // hot ints then cold ints
  double* d_dbl = nullptr;
  int rs = 0, smem_warp = 0;
  DevBuf queue[2], counters, save, resume, nst, nni, nje, status, stats;
  size_t cap = 0;
  static constexpr int kGraphs = 4;  // a few argument sets alternate (e.g. fallback list and judge sample)
  cudaGraphExec_t graph[kGraphs] = {};
  SubstepKey key[kGraphs] = {};
  int next_slot = 0;
  int warps = 0, occ = 0, blocks = 0, cold_in_smem = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

void solver_release(tng_chem* h) {
  SolverState* s = h->solver;
  if (!s) return;
  for (auto& g : s->graph)
    if (g) cudaGraphExecDestroy(g);
  if (s->d_int) cudaFree(s->d_int);
  if (s->d_dbl) cudaFree(s->d_dbl);
  if (s->d_coef) cudaFree(s->d_coef);
  for (DevBuf* b : {&s->queue[0], &s->queue[1], &s->counters, &s->save, &s->resume, &s->nst, &s->nni, &s->nje,
                    &s->status, &s->stats})
    b->release();
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  delete s;
  h->solver = nullptr;
}

static int ensure_tables(tng_chem* h) {
  if (!h->solver) h->solver = new SolverState();
  SolverState* s = h->solver;
  if (s->tables_ready) return TNG_OK;
  {
    const BdfCoef coef = make_coef();
    cudaError_t ce = cudaMalloc(&s->d_coef, sizeof(BdfCoef));
    if (ce == cudaSuccess) ce = cudaMemcpy(s->d_coef, &coef, sizeof(coef), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return cuda_error(ce, "BDF coefficients");
  }
  const MechOps* o = h->ops;
  const SvLayout& L = *o->sv_layout;
  if (L.size[SZ_NV] > 64)  // the warp holds a cell's state two entries per lane
    return set_error(TNG_ERR_ARG, "implicit solver: at most 63 species (%s has %d)", o->name, L.size[SZ_NS]);
  cudaError_t e;
  if ((e = cudaMalloc(&s->d_int, sizeof(int) * (L.nhi + L.nci))) != cudaSuccess) return cuda_error(e, "solver tables");
  if ((e = cudaMalloc(&s->d_dbl, sizeof(double) * L.nhd)) != cudaSuccess) return cuda_error(e, "solver tables");
  cudaMemcpy(s->d_int, o->sv_hi, sizeof(int) * L.nhi, cudaMemcpyHostToDevice);
  cudaMemcpy(s->d_int + L.nhi, o->sv_ci, sizeof(int) * L.nci, cudaMemcpyHostToDevice);
  cudaMemcpy(s->d_dbl, o->sv_hd[h->cfg.literal_mode], sizeof(double) * L.nhd, cudaMemcpyHostToDevice);
  s->dev.hd = s->d_dbl;
  s->dev.hi = s->d_int;
  s->dev.ci = s->d_int + L.nhi;
  s->dev.L = L;
  s->dev.mixed = h->cfg.precision == TNG_MIXED;
  const int nv = L.size[SZ_NV];
  s->rs = (nv % 2 == 0) ? nv + 1 : nv;
  s->smem_warp = warp_mem_doubles(L, s->rs);
  s->smem_warp = (s->smem_warp + 3) & ~3;
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  s->tables_ready = true;
  return TNG_OK;
}

// occ 2 (with 8 warps): launch bounds for two blocks per SM (registers capped at 128)
static BdfKernelFn bdf_kernel(const tng_chem* h, int warps, int occ = 1) {
  const SolverKernels* k = solver_kernels_for(h->ops->sk, h->cfg.precision == TNG_MIXED);
  if (warps == 8 && occ == 2) return k->bdf8_occ2;
  switch (warps) {
    case 2:
      return k->bdf2;
    case 8:
      return k->bdf8;
    default:
      return k->bdf4;
  }
}

static size_t block_smem(const SolverState* s, int warps, int cold) {
  return ((size_t)hot_smem_doubles(s->dev.L) + (cold ? (size_t)cold_smem_doubles(s->dev.L) : 0) +
          (size_t)warps * s->smem_warp) *
         sizeof(double);
}

static int configure_kernel(tng_chem* h, int warps, int occ, int* blocks_out) {
  SolverState* s = h->solver;
  // the Jacobian's term tables go to shared memory whenever the blocks still fit (the solver
  // kernels keep no stack, so L1 has nothing else to hold; the staged static BDF coefficients
  // take a further 1 KB)
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->cfg.device);
  s->cold_in_smem = (block_smem(s, warps, 1) + 1024) * occ <= (size_t)optin ? 1 : 0;
  const size_t smem = block_smem(s, warps, s->cold_in_smem);
  BdfKernelFn k = bdf_kernel(h, warps, occ);
  cudaError_t e = ensure_dynamic_smem((const void*)k, smem);
  if (e != cudaSuccess) return cuda_error(e, "solver shared memory");
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, warps * 32, smem);
  if (e != cudaSuccess) return cuda_error(e, "solver occupancy");
  if (per_sm < 1) return set_error(TNG_ERR_CUDA, "solver kernel does not fit on an SM (%zu B shared)", smem);
  *blocks_out = per_sm * h->sm_count;
  return TNG_OK;
}

// Totals of the per-cell counters: per-thread partials, warp sums, one global atomic per warp
// (one atomic per cell and counter serialised on the same addresses).
static __global__ void k_stats(const int* nst, const int* nni, const int* nje, const int* status, int64_t n,
                               unsigned long long* acc /* 5 + 2 + 16 */) {
  __shared__ unsigned long long hist[16];
  if (threadIdx.x < 16) hist[threadIdx.x] = 0;
  __syncthreads();
  unsigned long long s0 = 0, s1 = 0, s2 = 0, s3 = 0, m0 = 0, m1 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int a = nst[i], b = nni[i], c = nje[i];
    s0 += a, s1 += b, s2 += c, s3 += status[i] != 0;
    m0 = max(m0, (unsigned long long)a), m1 = max(m1, (unsigned long long)b);
    int bin = 0;
    for (int v = b; v > 0 && bin < 15; v >>= 1) ++bin;
    atomicAdd(&hist[bin], 1ULL);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    s3 += __shfl_xor_sync(0xffffffffu, s3, o);
    m0 = max(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (s0) atomicAdd(&acc[0], s0);
    if (s1) atomicAdd(&acc[1], s1);
    if (s2) atomicAdd(&acc[2], s2);
    if (s3) atomicAdd(&acc[3], s3);
    atomicMax(&acc[4], m0);
    atomicMax(&acc[5], m1);
  }
  __syncthreads();
  if (threadIdx.x < 16 && hist[threadIdx.x]) atomicAdd(&acc[8 + threadIdx.x], hist[threadIdx.x]);
}

int solver_prepare(tng_chem* h) {
  DeviceGuard g(h->cfg.device);
  return ensure_tables(h);
}

void solver_thermo(tng_chem* h, const double** th, double* tmid) {
  const SolverState* s = h->solver;
  *th = s->dev.hd + s->dev.L.hd[HD_TH];
  const int lm = h->cfg.literal_mode;
  *tmid = h->ops->sv_hd[lm][h->ops->sv_layout->hd[HD_SCAL] + SC_TMID];
}

// The implicit substep over ncells cells of a device state, or over the cells listed in
// list[0 .. *nlist) (device pointers; *nlist read on the device) when list is non-null.
int substep_run(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts, double dt, double p,
                int flags, const int* list, const int* nlist, int* cell_nst, int* cell_nni, int* cell_status,
                tng_substep_stats* stats);

}  // namespace tng

using namespace tng;

extern "C" int tng_substep_batch(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts, double dt,
                                 double p, int flags, int* cell_nst, int* cell_nni, int* cell_status,
                                 tng_substep_stats* stats) {
  return tng::substep_run(h, state, ncells, ld, dts, dt, p, flags, nullptr, nullptr, cell_nst, cell_nni, cell_status,
                          stats);
}

namespace tng {

int substep_run(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts, double dt, double p,
                int flags, const int* list, const int* nlist, int* cell_nst, int* cell_nni, int* cell_status,
                tng_substep_stats* stats) {
  if (!h) return set_error(TNG_ERR_ARG, "tng_substep_batch: null handle");
  if (ncells < 0 || ld < ncells) return set_error(TNG_ERR_ARG, "tng_substep_batch: need 0 <= ncells <= ld");
  if (ncells > (int64_t)0x7fffffff) return set_error(TNG_ERR_ARG, "tng_substep_batch: at most 2^31-1 cells");
  if (ncells > 0 && !state) return set_error(TNG_ERR_ARG, "tng_substep_batch: null state");
  if (!dts && !(dt >= 0.0)) return set_error(TNG_ERR_ARG, "tng_substep_batch: dt must be >= 0");
  if (!(p > 0.0)) return set_error(TNG_ERR_ARG, "tng_substep_batch: pressure must be positive");
  if (flags != TNG_DEVICE_PTRS && flags != TNG_HOST_PTRS) return set_error(TNG_ERR_ARG, "tng_substep_batch: bad flags");
  if (flags == TNG_HOST_PTRS && (cell_nst || cell_nni || cell_status))
    return set_error(TNG_ERR_ARG, "tng_substep_batch: per-cell arrays need device pointers");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (ncells == 0) return TNG_OK;
  DeviceGuard g(h->cfg.device);
  int rc = ensure_tables(h);
  if (rc) return rc;
  SolverState* s = h->solver;
  const int nv = h->ops->ns + 1;
  cudaError_t e;
  // host arrays: stage through device buffers (the staging buffers of the rate path)
  double* dstate = state;
  const double* ddts = dts;
  if (flags == TNG_HOST_PTRS) {
    if (!h->bufs[4].reserve((size_t)nv * ncells * sizeof(double)))
      return set_error(TNG_ERR_CUDA, "tng_substep_batch: device state allocation failed");
    dstate = (double*)h->bufs[4].ptr;
    e = cudaMemcpy2DAsync(dstate, ncells * sizeof(double), state, ld * sizeof(double), ncells * sizeof(double), nv,
                          cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_error(e, "state host->device");
    if (dts) {
      if (!h->bufs[5].reserve(ncells * sizeof(double))) return set_error(TNG_ERR_CUDA, "dt allocation failed");
      cudaMemcpyAsync(h->bufs[5].ptr, dts, ncells * sizeof(double), cudaMemcpyHostToDevice, h->stream);
      ddts = (const double*)h->bufs[5].ptr;
    }
  }
  const int64_t dld = flags == TNG_HOST_PTRS ? ncells : ld;
  // scratch
  const int budget = h->cfg.pass_budget > 0 ? h->cfg.pass_budget : 0x7fffffff;
  const int passes = budget == 0x7fffffff ? 1 : std::max(2, h->cfg.max_passes > 0 ? h->cfg.max_passes : 8);
  const int warps = (h->cfg.solver_warps == 2 || h->cfg.solver_warps == 4) ? h->cfg.solver_warps : 8;
  const int occ = (warps == 8 && h->cfg.solver_occupancy == 2) ? 2 : 1;
  const int save_stride = ((kQmax + 2) * nv + 16 + 3) & ~3;
  bool ok = s->counters.reserve(64 * sizeof(int)) && s->queue[0].reserve(ncells * sizeof(int)) &&
            s->queue[1].reserve(ncells * sizeof(int)) && s->resume.reserve(ncells * sizeof(int)) &&
            s->nst.reserve(ncells * sizeof(int)) && s->nni.reserve(ncells * sizeof(int)) &&
            s->nje.reserve(ncells * sizeof(int)) && s->status.reserve(ncells * sizeof(int)) &&
            s->stats.reserve(32 * sizeof(unsigned long long));
  if (ok && passes > 1) ok = s->save.reserve((size_t)ncells * save_stride * sizeof(double));
  if (!ok) return set_error(TNG_ERR_CUDA, "tng_substep_batch: scratch allocation for %lld cells failed", (long long)ncells);
  if (s->warps != warps || s->occ != occ) {
    if ((rc = configure_kernel(h, warps, occ, &s->blocks))) return rc;
    s->warps = warps;
    s->occ = occ;
  }
  int* nst = cell_nst ? cell_nst : (int*)s->nst.ptr;
  int* nni = cell_nni ? cell_nni : (int*)s->nni.ptr;
  int* sts = cell_status ? cell_status : (int*)s->status.ptr;
  if (list && flags != TNG_DEVICE_PTRS) return set_error(TNG_ERR_ARG, "substep: cell lists need device pointers");
  SubstepKey key{dstate, ncells, dld, list, nlist, ddts, dt, p, warps, occ, budget, passes, nst, nni, sts};
  int slot = -1;
  for (int i = 0; i < SolverState::kGraphs; ++i)
    if (s->graph[i] && s->key[i] == key) slot = i;
  if (slot < 0) {
    slot = s->next_slot;
    s->next_slot = (s->next_slot + 1) % SolverState::kGraphs;
    if (s->graph[slot]) {
      cudaGraphExecDestroy(s->graph[slot]);
      s->graph[slot] = nullptr;
    }
    BdfLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.coef = s->d_coef;
    BdfArgs& a = L.a;
    a.tab = s->dev;
    a.state = dstate;
    a.ld = dld;
    a.dts = ddts;
    a.dt_scalar = dt;
    a.p = p;
    a.save = (double*)s->save.ptr;
    a.save_stride = save_stride;
    a.resume = (int*)s->resume.ptr;
    a.rtol = h->cfg.rtol;
    a.atol = h->cfg.atol;
    a.dgmax = 0.3;
    a.max_steps = h->cfg.max_steps;
    a.maxcor = 3;
    a.msbp = 20;
    a.nst = nst;
    a.nni = nni;
    a.nje = (int*)s->nje.ptr;
    a.status = sts;
    a.smem_warp = s->smem_warp;
    a.rs = s->rs;
    int* cnt = (int*)s->counters.ptr;  // [0..1] heads, [2..3] out counts
    const size_t smem = block_smem(s, warps, s->cold_in_smem);
    L.cold_in_smem = s->cold_in_smem;
    cudaStream_t st = h->stream;
    if ((e = ensure_dynamic_smem((const void*)bdf_kernel(h, warps, occ), smem)) != cudaSuccess)
      return cuda_error(e, "solver shared memory");
    cudaError_t pending = cudaGetLastError();  // an earlier asynchronous error is reported, not captured
    if (pending != cudaSuccess) return cuda_error(pending, "implicit substep (error pending before the graph capture)");
    cudaError_t first = cudaSuccess;            // the first error inside the capture, and where
    const char* where = "";
    auto note = [&](cudaError_t r, const char* w) {
      if (first == cudaSuccess && r != cudaSuccess) first = r, where = w;
    };
    note(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    note(cudaMemsetAsync(s->resume.ptr, 0, ncells * sizeof(int), st), "resume flags");
    for (int pass = 0; pass < passes; ++pass) {
      const int cur = pass & 1;
      a.head = cnt + cur;
      a.n_out = cnt + 2 + cur;
      k_reset_counters<<<1, 32, 0, st>>>(a.head, a.n_out);
      note(cudaGetLastError(), "counter reset");
      a.queue_in = pass == 0 ? list : (const int*)s->queue[cur ^ 1].ptr;
      a.queue_out = (int*)s->queue[cur].ptr;
      a.n_in = (int)ncells;
      L.n_in_dev = pass == 0 ? nlist : cnt + 2 + (cur ^ 1);
      a.budget = pass == passes - 1 ? 0x7fffffff : budget;
      bdf_kernel(h, warps, occ)<<<s->blocks, warps * 32, smem, st>>>(L);
      note(cudaGetLastError(), "solver kernel");
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    if (first != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaFuncAttributes fa{};
      cudaFuncGetAttributes(&fa, bdf_kernel(h, warps, occ));
      cudaGetLastError();
      return set_error(TNG_ERR_CUDA,
                       "solver graph capture, %s (%d blocks x %d threads, %zu B shared; kernel: %d registers, %zu B "
                       "static shared, %d B dynamic shared allowed, %d threads allowed): %s",
                       where, s->blocks, warps * 32, smem, fa.numRegs, fa.sharedSizeBytes, fa.maxDynamicSharedSizeBytes,
                       fa.maxThreadsPerBlock, cudaGetErrorString(first));
    }
    if (e != cudaSuccess) return cuda_error(e, "solver graph capture");
    e = cudaGraphInstantiate(&s->graph[slot], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_error(e, "solver graph instantiate");
    s->key[slot] = key;
  }
  if (stats && list) {
    // cells outside the list keep older counters: clear them so the statistics cover the list only
    for (int* q : {nst, nni, (int*)s->nje.ptr, sts}) cudaMemsetAsync(q, 0, ncells * sizeof(int), h->stream);
  }
  cudaEventRecord(s->ev0, h->stream);
  if ((e = cudaGraphLaunch(s->graph[slot], h->stream)) != cudaSuccess) return cuda_error(e, "solver graph launch");
  cudaEventRecord(s->ev1, h->stream);
  if (flags == TNG_HOST_PTRS) {
    e = cudaMemcpy2DAsync(state, ld * sizeof(double), dstate, ncells * sizeof(double), ncells * sizeof(double), nv,
                          cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return cuda_error(e, "state device->host");
  }
  if (stats) {
    unsigned long long* acc = (unsigned long long*)s->stats.ptr;
    cudaMemsetAsync(acc, 0, 32 * sizeof(unsigned long long), h->stream);
    k_stats<<<std::min<int64_t>(1184, (ncells + 255) / 256), 256, 0, h->stream>>>(nst, nni, (int*)s->nje.ptr, sts,
                                                                                  ncells, acc);
    unsigned long long hacc[32];
    int hc[4], hlist = 0;
    cudaMemcpyAsync(hacc, acc, sizeof(hacc), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(hc, s->counters.ptr, sizeof(hc), cudaMemcpyDeviceToHost, h->stream);
    if (list) cudaMemcpyAsync(&hlist, nlist, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_error(e, "implicit substep");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    stats->cells = list ? hlist : ncells;
    stats->steps = (int64_t)hacc[0];
    stats->newton_iters = (int64_t)hacc[1];
    stats->jacobians = (int64_t)hacc[2];
    stats->cells_failed = (int64_t)hacc[3];
    stats->max_steps_cell = (int)hacc[4];
    stats->max_newton_cell = (int)hacc[5];
    for (int b = 0; b < 16; ++b) stats->newton_hist[b] = (int)hacc[8 + b];
    stats->passes = passes;
    stats->ms = ms;
  } else if (flags == TNG_HOST_PTRS) {
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_error(e, "implicit substep");
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "implicit substep");
  return TNG_OK;
}

}  // namespace tng

extern "C" int tng_solver_rhs_jac(tng_chem* h, const double* state, int64_t ncells, int64_t ld, double p, double* rhs,
                                  double* jac) {
  if (!h || !state || !rhs) return set_error(TNG_ERR_ARG, "tng_solver_rhs_jac: null argument");
  if (ncells <= 0 || ld < ncells) return set_error(TNG_ERR_ARG, "tng_solver_rhs_jac: bad sizes");
  DeviceGuard g(h->cfg.device);
  int rc = ensure_tables(h);
  if (rc) return rc;
  SolverState* s = h->solver;
  const size_t smem = block_smem(s, 4, 0);
  const RhsJacFn kern = solver_kernels_for(h->ops->sk, h->cfg.precision == TNG_MIXED)->rhs_jac4;
  cudaError_t e = ensure_dynamic_smem((const void*)kern, smem);
  if (e != cudaSuccess) return cuda_error(e, "solver shared memory");
  const int blocks = (int)std::min<int64_t>((ncells + 3) / 4, 148 * 8);
  kern<<<blocks, 128, smem, h->stream>>>(s->dev, state, ld, (int)ncells, p, rhs, jac, s->smem_warp);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "tng_solver_rhs_jac");
  return TNG_OK;
}
