// tng_substep_batch_static: the implicit substep of tng_substep_batch (device pointers, one
// pass, no step budget) for callers that must not allocate device memory during the call.
//
// Who cannot allocate: a host CFD code that hands most of the GPU's memory to its own pool
// before the time loop starts, or that calls the chemistry from inside a region where a
// cudaMalloc would synchronise the device (and so stall its other streams) or could fail
// with out-of-memory half-way through a time step. tng_substep_batch grows per-cell scratch
// on demand; this entry point instead carves every byte it needs -- solver tables, per-cell
// counters, the work-stealing counter -- out of one file-scope __device__ array of fixed size.
//
// Limits and contract:
//   * at most kStaticMaxCells cells per call (TNG_ERR_ARG beyond that);
//   * the first call on a device does the set-up: the symbol address, the BDF coefficients
//     and the solver tables of EVERY built-in mechanism (both literal modes) into their own
//     fixed regions of the array. Those copies are synchronous,
//     so that first call should come before any stream capture the caller does. A later call
//     only selects its mechanism's region: it copies no tables, so calls of different
//     mechanisms can follow each other in any order (and a captured call stays valid);
//   * with n_failed non-null the call reads the failure count back and waits for the stream,
//     which a stream capture does not allow: n_failed must then be NULL (TNG_ERR_ARG);
//   * the scratch is one per device and process: two calls that overlap in time on the same
//     device (different streams, or different threads without ordering) race on it and give
//     wrong results. Calls must be ordered, e.g. all on one stream;
//   * what must start at zero (per-cell resume flags, the work-stealing head) is cleared on
//     the call's stream by every call, so consecutive calls need no caller action.
// Nothing here calls cudaMalloc, cudaMallocAsync, cudaFree or a routine that allocates.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "bdf_kernel.cuh"
#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

namespace {

constexpr int kStaticMaxCells = 1 << 18;
constexpr size_t kStaticTabBytes = (size_t)1 << 20;  // tables of all built-in mechanisms (~0.3 MB used)
constexpr int kStaticMaxMechs = 16;
constexpr int kStaticMaxDevices = 64;

// byte offsets inside the scratch array (each region 256-byte aligned)
constexpr size_t kOffTab = 0;
constexpr size_t kOffCtr = kOffTab + kStaticTabBytes;                               // head, n_out, n_failed
constexpr size_t kOffCells = kOffCtr + 256;                                         // 6 int arrays of kStaticMaxCells
constexpr size_t kScratchBytes = kOffCells + sizeof(int) * 6 * (size_t)kStaticMaxCells;  // ~7.3 MB
static_assert(kOffCtr % 256 == 0 && kOffCells % 256 == 0, "alignment");

static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

// where one mechanism's tables sit in the table area (byte offsets)
struct StaticTab {
  const MechOps* ops = nullptr;
  size_t hd[2] = {0, 0};  // hot doubles per literal mode
  size_t ints = 0;        // hot ints, then cold ints
};

struct StaticDev {
  bool ready = false;
  unsigned char* base = nullptr;
  size_t coef = 0;  // the BDF coefficients (byte offset)
  StaticTab tab[kStaticMaxMechs];
  int ntab = 0;
};
StaticDev g_dev[kStaticMaxDevices];
std::mutex g_setup_mutex;

__global__ void k_count_failed(const int* status, int n, int* n_failed) {
  int c = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += status[i] != 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(n_failed, c);
}

int static_setup(int device, StaticDev** out) {
  if (device < 0 || device >= kStaticMaxDevices) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: device index");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  StaticDev& d = g_dev[device];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return cuda_error(e, "tng_substep_batch_static: scratch symbol address");
    // the BDF coefficients, then every built-in mechanism's tables into its own region, packed
    // in registry order
    unsigned char* base = (unsigned char*)p;
    size_t off = kOffTab;
    int nt = 0;
    auto place = [&](const void* src, size_t bytes, size_t* at) -> int {
      if (off + bytes > kOffTab + kStaticTabBytes)
        return set_error(TNG_ERR_ARG, "tng_substep_batch_static: the mechanism tables exceed the static table area");
      const cudaError_t ce = cudaMemcpy(base + off, src, bytes, cudaMemcpyHostToDevice);
      if (ce != cudaSuccess) return cuda_error(ce, "tng_substep_batch_static: solver tables");
      *at = off;
      off += (bytes + 255) & ~(size_t)255;
      return TNG_OK;
    };
    const BdfCoef coef = make_coef();
    if (int rc = place(&coef, sizeof(coef), &d.coef)) return rc;
    for (const MechOps* const* m = all_mechanisms(); *m; ++m) {
      if (nt == kStaticMaxMechs) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: too many mechanisms");
      const MechOps* o = *m;
      const SvLayout& L = *o->sv_layout;
      StaticTab& t = d.tab[nt];
      t.ops = o;
      int rc = TNG_OK;
      for (int lm = 0; lm < 2 && !rc; ++lm) rc = place(o->sv_hd[lm], sizeof(double) * L.nhd, &t.hd[lm]);
      if (!rc) rc = place(o->sv_hi, sizeof(int) * L.nhi, &t.ints);
      size_t cold = 0;
      if (!rc) rc = place(o->sv_ci, sizeof(int) * L.nci, &cold);
      if (rc) return rc;
      if (cold != t.ints + ((sizeof(int) * L.nhi + 255) & ~(size_t)255))
        return set_error(TNG_ERR_STATE, "tng_substep_batch_static: table placement");
      ++nt;
    }
    d.ntab = nt;
    d.base = base;
    d.ready = true;  // only once every copy has succeeded
  }
  *out = &d;
  return TNG_OK;
}

}  // namespace
}  // namespace tng

using namespace tng;

extern "C" int tng_substep_batch_static(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts,
                                        double dt, double p, int* n_failed) {
  if (!h) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: null handle");
  if (ncells < 0 || ld < ncells) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: need 0 <= ncells <= ld");
  if (ncells > kStaticMaxCells)
    return set_error(TNG_ERR_ARG, "tng_substep_batch_static: %lld cells exceed the static limit of %d per call",
                     (long long)ncells, kStaticMaxCells);
  if (ncells > 0 && !state) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: null state");
  if (!dts && !(dt >= 0.0)) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: dt must be >= 0");
  if (!(p > 0.0)) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: pressure must be positive");
  const MechOps* o = h->ops;
  const SvLayout& L = *o->sv_layout;
  if (n_failed) *n_failed = 0;
  if (ncells == 0) return TNG_OK;
  DeviceGuard g(h->cfg.device);
  cudaStream_t st = h->stream;
  cudaError_t e;
  if (n_failed) {  // the count is read back synchronously, which a stream capture forbids
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess) return cuda_error(e, "tng_substep_batch_static");
    if (cs != cudaStreamCaptureStatusNone)
      return set_error(TNG_ERR_ARG, "tng_substep_batch_static: n_failed must be NULL while the stream is captured");
  }
  StaticDev* d = nullptr;
  int rc = static_setup(h->cfg.device, &d);
  if (rc) return rc;
  const StaticTab* tab = nullptr;
  for (int i = 0; i < d->ntab; ++i)
    if (d->tab[i].ops == o) tab = &d->tab[i];
  if (!tab) return set_error(TNG_ERR_ARG, "tng_substep_batch_static: %s is not a built-in mechanism", o->name);
  const double* tab_d = (const double*)(d->base + tab->hd[h->cfg.literal_mode == 1 ? 1 : 0]);
  const int* tab_i = (const int*)(d->base + tab->ints);
  const int* tab_c = (const int*)(d->base + tab->ints + ((sizeof(int) * L.nhi + 255) & ~(size_t)255));
  int* ctr = (int*)(d->base + kOffCtr);
  int* cells = (int*)(d->base + kOffCells);
  const int warps = (h->cfg.solver_warps == 2 || h->cfg.solver_warps == 4) ? h->cfg.solver_warps : 8;
  BdfLaunch Lh;
  std::memset(&Lh, 0, sizeof(Lh));
  Lh.coef = (const BdfCoef*)(d->base + d->coef);
  BdfArgs& a = Lh.a;
  a.tab.hd = tab_d;
  a.tab.hi = tab_i;
  a.tab.ci = tab_c;
  a.tab.L = L;
  a.tab.mixed = h->cfg.precision == TNG_MIXED;
  const int nv = L.size[SZ_NV];
  a.rs = (nv % 2 == 0) ? nv + 1 : nv;
  a.smem_warp = (warp_mem_doubles(L, a.rs) + 3) & ~3;
  const size_t smem = ((size_t)hot_smem_doubles(L) + (size_t)warps * a.smem_warp) * sizeof(double);
  const SolverKernels* sk = solver_kernels_for(o->sk, a.tab.mixed);
  const BdfKernelFn kern = warps == 2 ? sk->bdf2 : warps == 4 ? sk->bdf4 : sk->bdf8;
  e = ensure_dynamic_smem((const void*)kern, smem);
  if (e != cudaSuccess) return cuda_error(e, "tng_substep_batch_static: shared memory");
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem);
  if (e != cudaSuccess) return cuda_error(e, "tng_substep_batch_static: occupancy");
  if (per_sm < 1) return set_error(TNG_ERR_CUDA, "tng_substep_batch_static: kernel does not fit on an SM");
  const int n = (int)ncells;
  a.state = state;
  a.ld = ld;
  a.dts = dts;
  a.dt_scalar = dt;
  a.p = p;
  a.queue_in = nullptr;
  a.n_in = n;
  a.head = ctr;
  a.n_out = ctr + 1;
  a.resume = cells;
  a.nst = cells + (size_t)kStaticMaxCells;
  a.nni = cells + 2 * (size_t)kStaticMaxCells;
  a.nje = cells + 3 * (size_t)kStaticMaxCells;
  a.status = cells + 4 * (size_t)kStaticMaxCells;
  a.queue_out = cells + 5 * (size_t)kStaticMaxCells;
  a.save = nullptr;  // one pass without a step budget never saves integrator state
  a.save_stride = 0;
  a.budget = 0x7fffffff;
  a.rtol = h->cfg.rtol;
  a.atol = h->cfg.atol;
  a.dgmax = 0.3;
  a.max_steps = h->cfg.max_steps;
  a.maxcor = 3;
  a.msbp = 20;
  Lh.n_in_dev = nullptr;
  // zero state: resume flags of the cells in this call, head / n_out / failure count
  cudaMemsetAsync(a.resume, 0, sizeof(int) * (size_t)n, st);
  cudaMemsetAsync(ctr, 0, 4 * sizeof(int), st);
  kern<<<per_sm * h->sm_count, warps * 32, smem, st>>>(Lh);
  if (n_failed) {
    k_count_failed<<<std::min(1184, (n + 255) / 256), 256, 0, st>>>(a.status, n, ctr + 2);
    int hcount = 0;
    cudaMemcpyAsync(&hcount, ctr + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "tng_substep_batch_static");
    *n_failed = hcount;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "tng_substep_batch_static");
  return TNG_OK;
}
