// K4: surrogate inference on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One launch evaluates every network of the surrogate (the ensemble members and the error gate)
// on the same cells. Persistent CTAs (two per SM) walk tiles of 128 cells. For each tile:
//   1. features: the 256 threads split each cell's species between two threads, issue all their
//      FP64 state loads at once (one memory latency per tile, not one per species), form the
//      density, temperature and the normalised inputs, and keep them packed as BF16 in registers;
//   2. for each network, the features are written into shared memory (UMMA canonical K-major
//      layout, 8-row x 16-byte core matrices) and every layer is D[128 x N] = H[128 x K] * W^T on
//      tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator in tensor memory); one elected
//      thread issues the MMAs, weights stream from global memory (L2-resident, shared by all
//      CTAs) into a two-stage shared-memory ring with cp.async.bulk + mbarrier transaction
//      counts, and the next layer's (next network's, next tile's) first chunk is fetched while the
//      epilogue runs; tcgen05.commit releases ring stages;
//   3. the epilogue (8 warps, two per tensor-memory lane quarter) reads D with tcgen05.ld, adds
//      the bias, applies GELU and writes the next layer's BF16 operand back into shared memory;
//      the last layer's FP32 outputs go to the network's output array.
// Every wait is bounded: on expiry the CTA records an error code and stops issuing work.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tng {

constexpr int kInferRows = 128;
constexpr int kInferThreads = 256;  // 8 warps: two per TMEM lane quarter
constexpr int kWChunkK = 32;   // K width of one streamed weight chunk (two MMAs)
constexpr int kWStages = 2;    // weight stages: one chunk in flight ahead of the MMA
constexpr int kMaxLayers = 9;
constexpr int kMaxNets = 5;    // ensemble members and the error gate
constexpr int kFeatSpecies = 24;  // species per feature thread (two threads per cell): ns <= 48

// One network of the launch: hidden layers of the launch's shared shape, its own last layer.
struct InferNet {
  const __nv_bfloat16* wpack;   // all layers, chunked canonical layout
  long long w_off[kMaxLayers];  // element offset of layer l in wpack
  const float* bias;            // all layers, fan_out entries each
  int b_off[kMaxLayers];        // offset of layer l's bias in `bias`
  int out_pad;                  // width of the last layer (multiple of 16)
  float* out;                   // [ncells x out_pad] FP32 (normalised predictions)
};

struct InferArgs {
  const double* state;  // species-major [v*ld + cell]
  long long ld;
  int ncells;
  const double* dts;  // per-cell dt or null
  double dt_scalar;
  double logp;        // log(pressure)
  int ns;             // species count
  int bath;           // species index left out of the inputs (the bath gas)
  int n_in, in_pad, hidden, nlin;
  const float* fmean;  // feature normalisation, n_in entries
  const float* fistd;  // 1/std
  int nnets;
  InferNet net[kMaxNets];
  int* error;  // non-zero after a timed-out wait
  // test hook: polls before a wait gives up (0: the default 2^24), and fault = 1 withholds the
  // first layer's completion signal of each CTA's first tile so that the epilogue's wait runs
  // out (the MMAs themselves run and are drained as usual)
  int wait_limit;
  int fault;
};

// Raw network input i of a cell (shared by the training features, the inference kernel and the
// range check): 0 T; 1 log P; 2 .. ns log10 Y_k; ns+1 log10 dt; ns+2 .. 2ns Y_k -- the species
// in mechanism order without the bath gas, once on a log scale (trace radicals) and once linear
// (heat release is linear in the mass fractions). n_in = 2 ns + 1.
__device__ __forceinline__ float sur_raw_input(int i, int ns, int bath, const double* __restrict__ state, long long ld,
                                               int cell, double irho, double T, double logp, double dt) {
  if (i == 0) return (float)T;
  if (i == 1) return (float)logp;
  if (i == ns + 1) return (float)log10(fmax(dt, 1e-30));
  if (i >= 2 * ns + 1) return 0.f;
  const bool lin = i > ns + 1;
  int k = lin ? i - ns - 2 : i - 2;
  if (k >= bath) ++k;
  const double y = state[(long long)k * ld + cell] * irho;  // irho = 1 / rho
  // the logarithm in FP32: the feature is rounded to FP32 (and to BF16 for the network) anyway
  return lin ? (float)y : log10f(fmaxf((float)y, 1e-30f));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// canonical K-major, no swizzle: byte offset of element (r, k) in a [R x K] bf16 operand
__device__ __forceinline__ uint32_t canon_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;              // base offset 0, layout SWIZZLE_NONE
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both operands K-major
__device__ __forceinline__ uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

constexpr int kWaitPolls = 1 << 24;

// bounded parity wait; returns false after `limit` unsuccessful polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int limit = kWaitPolls) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu_fast(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * x * (1.0f + t);
}

// shared-memory plan (bytes): A operand (128 x 256 bf16 = 64 KB), two weight stages of
// 256 x 32 bf16 (16 KB each), barriers and the TMEM address: 96 KB, two CTAs per SM (their
// phases -- features, MMA, epilogue -- overlap), 2 x 256 TMEM columns.
constexpr int kSmemA = kInferRows * 256 * 2;
constexpr int kSmemStage = 256 * kWChunkK * 2;
constexpr int kInferSmem = kSmemA + kWStages * kSmemStage + 128;

__device__ __forceinline__ void st_bf16(uint8_t* sA, int row, int col, int K, __nv_bfloat16 v) {
  *reinterpret_cast<__nv_bfloat16*>(sA + canon_off(row, col, K)) = v;
}

__global__ void __launch_bounds__(kInferThreads, 2) k_mlp_infer(const InferArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* sA = sm;
  uint8_t* sW = sm + kSmemA;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kSmemA + kWStages * kSmemStage);
  // bars[0..S): stage full, bars[S..2S): stage free, bars[2S]: layer done
  uint64_t* bar_full = bars;
  uint64_t* bar_free = bars + kWStages;
  uint64_t* bar_done = bars + 2 * kWStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kWStages + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  __shared__ double s_part[2][kInferRows];  // the two halves of each cell's density
  if (tid == 0) {
    for (int i = 0; i < 2 * kWStages + 1; ++i) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int wlim = a.wait_limit > 0 ? a.wait_limit : kWaitPolls;
  // thread 0 only: parities, pending commits and copies per stage; chunks issued so far (stage =
  // gc % kWStages); chunks of the coming layer already issued (pre) from gc = pre_base
  uint32_t ph_full[kWStages] = {}, ph_free[kWStages] = {}, ph_done = 0;
  int stage_busy[kWStages] = {}, inflight[kWStages] = {};
  int gc = 0, pre = 0, pre_base = 0;
  int err = 0;
  // issue the bulk copy of weight chunk c of layer l of network ni into the next stage (thread 0)
  auto issue = [&](int ni, int l, int c) {
    const int K = l == 0 ? a.in_pad : a.hidden;
    const int N = l == a.nlin - 1 ? a.net[ni].out_pad : a.hidden;
    const int s = gc % kWStages;
    ++gc;
    if (stage_busy[s]) {  // wait for the MMA that read this stage
      if (!mbar_wait(&bar_free[s], ph_free[s], wlim)) err = 1;
      ph_free[s] ^= 1;
      stage_busy[s] = 0;
    }
    const int kc = min(kWChunkK, K - c * kWChunkK);
    const uint32_t bytes = (uint32_t)N * kc * 2;
    mbar_expect_tx(&bar_full[s], bytes);
    bulk_g2s(sW + s * kSmemStage, a.net[ni].wpack + a.net[ni].w_off[l] + (long long)c * N * kWChunkK, bytes,
             &bar_full[s]);
    inflight[s] = 1;
  };
  // this thread's share of a cell's inputs, normalised, kept as BF16 for every network: species
  // k0 + j (j < kn) as (log10 Y, Y) pairs; thread part 0 also holds T, log P and log10 dt
  const int row = tid & (kInferRows - 1), part = tid >> 7;
  const int half = (a.ns + 1) >> 1, k0 = part * half, kn = min(half, a.ns - k0);
  __nv_bfloat162 fsp[kFeatSpecies];
  __nv_bfloat162 fx0 = __floats2bfloat162_rn(0.f, 0.f), fx1 = fx0;
  // column of species k's log feature (k != bath); its linear feature is ns columns further
  auto log_col = [&](int k) { return 2 + (k < a.bath ? k : k - 1); };
  // the packed inputs into A (layer 0's operand, K = in_pad), zero padding included
  auto write_inputs = [&]() {
    const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
#pragma unroll
    for (int j = 0; j < kFeatSpecies; ++j) {
      const int k = k0 + j;
      if (j < kn && k != a.bath) {
        st_bf16(sA, row, log_col(k), a.in_pad, __low2bfloat16(fsp[j]));
        st_bf16(sA, row, log_col(k) + a.ns, a.in_pad, __high2bfloat16(fsp[j]));
      }
    }
    if (part == 0) {
      st_bf16(sA, row, 0, a.in_pad, __low2bfloat16(fx0));
      st_bf16(sA, row, 1, a.in_pad, __high2bfloat16(fx0));
      st_bf16(sA, row, a.ns + 1, a.in_pad, __low2bfloat16(fx1));
    } else {
      for (int i = a.n_in; i < a.in_pad; ++i) st_bf16(sA, row, i, a.in_pad, z);
    }
  };
  const int ntiles = (a.ncells + kInferRows - 1) / kInferRows;
  for (int tile = blockIdx.x; tile < ntiles && !err; tile += gridDim.x) {
    // ---- 1. features of the tile's cells (once for all networks)
    {
      const int cell = tile * kInferRows + row;
      const bool live = cell < a.ncells;
      double x[kFeatSpecies];
#pragma unroll
      for (int j = 0; j < kFeatSpecies; ++j) x[j] = (live && j < kn) ? a.state[(long long)(k0 + j) * a.ld + cell] : 0.0;
      const double xT = (live && part == 0) ? a.state[(long long)a.ns * a.ld + cell] : 0.0;
      const double dt = (live && part == 0) ? (a.dts ? a.dts[cell] : a.dt_scalar) : 1.0;
      double ps = 0.0;
#pragma unroll
      for (int j = 0; j < kFeatSpecies; ++j) ps += x[j];
      s_part[part][row] = ps;
      __syncthreads();
      const double rho = live ? s_part[0][row] + s_part[1][row] : 1.0;
      const double irho = 1.0 / rho;
#pragma unroll
      for (int j = 0; j < kFeatSpecies; ++j) {
        const int k = k0 + j;
        float fl = 0.f, fn = 0.f;
        if (live && j < kn && k != a.bath) {
          const int i = log_col(k);
          const double y = x[j] * irho;
          // the logarithm in FP32: the feature is rounded to FP32 (and to BF16 for the network) anyway
          fl = (log10f(fmaxf((float)y, 1e-30f)) - a.fmean[i]) * a.fistd[i];
          fn = ((float)y - a.fmean[i + a.ns]) * a.fistd[i + a.ns];
        }
        fsp[j] = __floats2bfloat162_rn(fl, fn);
      }
      if (part == 0) {
        float f0 = 0.f, f1 = 0.f, f2 = 0.f;
        if (live) {
          f0 = ((float)(xT / rho) - a.fmean[0]) * a.fistd[0];
          f1 = ((float)a.logp - a.fmean[1]) * a.fistd[1];
          f2 = ((float)log10(fmax(dt, 1e-30)) - a.fmean[a.ns + 1]) * a.fistd[a.ns + 1];
        }
        fx0 = __floats2bfloat162_rn(f0, f1);
        fx1 = __floats2bfloat162_rn(f2, 0.f);
      }
    }
    // ---- 2./3. networks and their layers
    for (int ni = 0; ni < a.nnets && !err; ++ni) {
      const InferNet& net = a.net[ni];
      write_inputs();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int l = 0; l < a.nlin && !err; ++l) {
        const int K = l == 0 ? a.in_pad : a.hidden;
        const int N = l == a.nlin - 1 ? net.out_pad : a.hidden;
        const int nchunk = (K + kWChunkK - 1) / kWChunkK;
        if (tid == 0) {
          const uint32_t idesc = umma_idesc(kInferRows, N);
          const uint32_t a_sbo = (uint32_t)K * 16;
          // chunk c sits in stage (base + c) % S; after chunk c's MMA is queued the copies of the
          // chunks up to c + S - 1 are issued, so they load while the tensor core works
          const int base = pre ? pre_base : gc;
          int issued = pre;
          pre = 0;
          if (issued == 0) issue(ni, l, issued++);
          for (int c = 0; c < nchunk && !err; ++c) {
            const int s = (base + c) % kWStages;
            const int kc = min(kWChunkK, K - c * kWChunkK);
            if (!mbar_wait(&bar_full[s], ph_full[s], wlim)) err = 1;
            ph_full[s] ^= 1;
            inflight[s] = 0;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t wbase = smem_u32(sW + s * kSmemStage);
            const uint32_t abase = smem_u32(sA);
            for (int kk = 0; kk < kc; kk += 16) {
              const int kg = c * kWChunkK + kk;
              const uint64_t ad = umma_desc(abase + (uint32_t)(kg >> 3) * 128, 128, a_sbo);
              const uint64_t bd = umma_desc(wbase + (uint32_t)(kk >> 3) * 128, 128, (uint32_t)kc * 16);
              umma_bf16(tmem, ad, bd, idesc, (c > 0 || kk > 0) ? 1u : 0u);
            }
            umma_commit(&bar_free[s]);
            stage_busy[s] = 1;
            while (issued < nchunk && issued < c + kWStages) issue(ni, l, issued++);
          }
          if (!(a.fault == 1 && ni == 0 && l == 0 && tile == (int)blockIdx.x)) umma_commit(bar_done);
        }
        // epilogue: one lane per warp polls the layer barrier, the warp follows
        bool ok = true;
        if ((tid & 31) == 0) ok = mbar_wait(bar_done, ph_done, wlim);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        ph_done ^= 1;
        if (!ok) err = 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // after a timed-out wait the layer's MMAs may still read the A operand: no epilogue
        if (__syncthreads_or(err)) {
          err = 1;
          break;
        }
        // the next layer's (next network's, next tile's) first chunks load during the epilogue
        if (tid == 0) {
          int nn = ni, nl = l + 1;
          if (nl == a.nlin) nl = 0, nn = ni + 1;
          if (nn == a.nnets) nn = 0;
          const bool more = l + 1 < a.nlin || ni + 1 < a.nnets || tile + (int)gridDim.x < ntiles;
          if (more) {
            const int nk = ((nl == 0 ? a.in_pad : a.hidden) + kWChunkK - 1) / kWChunkK;
            pre_base = gc;
            pre = min(nk, kWStages - 1);
            for (int c = 0; c < pre; ++c) issue(nn, nl, c);
          }
        }
        // warps w and w + 4 read the same TMEM lane quarter (rows), alternate 32-column groups
        const float* bl = net.bias + net.b_off[l];
        const int erow = (warp & 3) * 32 + (tid & 31);
        const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
        const bool last = l == a.nlin - 1;
        const int cell = tile * kInferRows + erow;
        for (int c0 = (warp >> 2) * 32; c0 < N; c0 += 64) {
          float v[32];
          tmem_ld32(trow + (uint32_t)c0, v);
          const int nc = min(32, N - c0);
          if (last) {
            if (cell < a.ncells) {
              float* o = net.out + (long long)cell * net.out_pad + c0;
              for (int i = 0; i < nc; ++i) o[i] = v[i] + __ldg(bl + c0 + i);
            }
          } else {
            const float4* b4 = reinterpret_cast<const float4*>(bl + c0);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float4 ba = __ldg(b4 + 2 * q), bb = __ldg(b4 + 2 * q + 1);
              const float bq[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
              float xq[8];
#pragma unroll
              for (int i = 0; i < 8; ++i) xq[i] = gelu_fast(v[q * 8 + i] + bq[i]);
              __nv_bfloat162 p0 = __floats2bfloat162_rn(xq[0], xq[1]);
              __nv_bfloat162 p1 = __floats2bfloat162_rn(xq[2], xq[3]);
              __nv_bfloat162 p2 = __floats2bfloat162_rn(xq[4], xq[5]);
              __nv_bfloat162 p3 = __floats2bfloat162_rn(xq[6], xq[7]);
              uint4 u;
              u.x = *reinterpret_cast<uint32_t*>(&p0);
              u.y = *reinterpret_cast<uint32_t*>(&p1);
              u.z = *reinterpret_cast<uint32_t*>(&p2);
              u.w = *reinterpret_cast<uint32_t*>(&p3);
              *reinterpret_cast<uint4*>(sA + canon_off(erow, c0 + q * 8, a.hidden)) = u;
            }
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        err = __syncthreads_or(err);
      }
    }
  }
  // drain: weight copies still in flight (after an error) and the last commits on the stage
  // barriers must complete before the CTA exits; every wait is bounded
  if (tid == 0) {
    for (int s = 0; s < kWStages; ++s) {
      if (inflight[s] && !mbar_wait(&bar_full[s], ph_full[s])) err = 1;
      if (stage_busy[s]) {
        if (!mbar_wait(&bar_free[s], ph_free[s])) err = 1;
        ph_free[s] ^= 1;
      }
    }
  }
  if (err && tid == 0 && a.error) atomicExch(a.error, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem));
}

}  // namespace tng
