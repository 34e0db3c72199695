// K4: surrogate inference on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One launch evaluates every network of the surrogate (the ensemble members and the error gate)
// on the same cells. Persistent CTAs (two per SM) walk tiles of 128 cells; every layer of every
// network is one step D[128 x N] = H[128 x K] * W^T on tcgen05.mma (kind::f16, BF16 operands,
// FP32 accumulator in tensor memory, A in shared memory in the UMMA canonical K-major layout of
// 8-row x 16-byte core matrices). The warps of a CTA have three roles:
//   * the weight producer (one warp, one lane) streams the weights of every step, in step order,
//     from global memory (L2-resident, shared by all CTAs) through a three-stage shared-memory
//     ring of 32-wide K chunks with cp.async.bulk and mbarrier transaction counts; it runs up to
//     three chunks ahead of the tensor core, across layers, networks and tiles;
//   * the MMA issuer (one warp, one lane) waits for a step's A operand, then for each chunk, issues
//     its MMAs, releases the chunk's stage with tcgen05.commit, and after the last chunk commits
//     the accumulator to the epilogue;
//   * eight feature/epilogue warps: per tile they form the features (the two threads of a cell,
//     lanes 2r and 2r+1 of one warp, split its species, issue all their FP64 state loads at once
//     and combine the density by a shuffle) and keep them packed as BF16 in registers; per step
//     they read D with tcgen05.ld (two warps per tensor-memory lane quarter), add the bias, apply
//     GELU and write the next step's A operand (or write the last layer's FP32 outputs and then
//     the next network's or tile's features), and signal the MMA issuer.
// So the tensor core never waits for a weight copy that the producer could have issued earlier,
// and with two CTAs per SM one CTA's epilogue overlaps the other's MMAs. Every wait is bounded:
// on expiry the waiting role records an error in shared memory, every role stops at its next
// wait, the issued copies and MMAs drain, and the CTA reports the error.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tng {

constexpr int kInferRows = 128;
constexpr int kEpiThreads = 256;                 // 8 feature/epilogue warps: two per TMEM lane quarter
constexpr int kInferThreads = kEpiThreads + 64;  // + the weight producer warp and the MMA warp
constexpr int kWChunkK = 32;   // K width of one streamed weight chunk (two MMAs)
constexpr int kWStages = 3;    // weight stages of the ring
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

// bounded parity wait; returns false after `limit` unsuccessful polls, or (with a flag) as soon
// as another role has recorded an error
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int limit = kWaitPolls,
                                          const volatile int* stop = nullptr) {
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
    if (stop && (it & 63) == 63 && *stop) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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

// Packed FP32 pairs (sm_100 f32x2 instructions: one FMA / MUL / ADD for two values; each lane is
// rounded as the scalar instruction would round it). Element 0 in the low 32 bits.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float x, float y) {
  return (f32x2)__float_as_uint(x) | ((f32x2)__float_as_uint(y) << 32);
}
__device__ __forceinline__ float f2_lo(f32x2 v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float f2_hi(f32x2 v) { return __uint_as_float((unsigned)(v >> 32)); }
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// GELU in its tanh form, 0.5 x (1 + tanh(u)), u = sqrt(2/pi) (x + 0.044715 x^3), of two values:
// u = x (c0 + c1 x^2) with c0 = sqrt(2/pi), c1 = 0.044715 sqrt(2/pi), and 0.5 x + 0.5 x tanh(u);
// five packed instructions and two tanh.approx for the pair
__device__ __forceinline__ f32x2 gelu2(f32x2 x) {
  const f32x2 c0 = f2_pack(0.7978845608028654f, 0.7978845608028654f);
  const f32x2 c1 = f2_pack(0.035677408136300125f, 0.035677408136300125f);
  const f32x2 hf = f2_pack(0.5f, 0.5f);
  const f32x2 u = f2_mul(x, f2_fma(f2_mul(x, x), c1, c0));
  float t0, t1;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t0) : "f"(f2_lo(u)));
  asm("tanh.approx.f32 %0, %1;" : "=f"(t1) : "f"(f2_hi(u)));
  const f32x2 h = f2_mul(x, hf);
  return f2_fma(h, f2_pack(t0, t1), h);
}

// shared-memory plan (bytes): A operand (128 x 256 bf16 = 64 KB), three weight stages of
// 256 x 32 bf16 (16 KB each), barriers, the TMEM address and the error flag: 112.1 KB; two CTAs
// per SM (with the per-block reserve, 226 KB of the SM's 228 KB), 2 x 256 TMEM columns.
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
  // bars[0..S): stage full; [S..2S): stage free; [2S]: accumulator full (MMA -> epilogue);
  // [2S+1]: A operand written and accumulator drained (epilogue -> MMA); [2S+2]: MMA drain
  uint64_t* bar_full = bars;
  uint64_t* bar_free = bars + kWStages;
  uint64_t* bar_acc = bars + 2 * kWStages;
  uint64_t* bar_ain = bars + 2 * kWStages + 1;
  uint64_t* bar_drain = bars + 2 * kWStages + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kWStages + 3);
  volatile int* s_err = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int kProdWarp = kEpiThreads / 32, kMmaWarp = kProdWarp + 1;
  if (tid == 0) {
    for (int i = 0; i < kWStages; ++i) {
      mbar_init(&bar_full[i], 1);
      mbar_init(&bar_free[i], 1);
    }
    mbar_init(bar_acc, 1);
    mbar_init(bar_ain, kEpiThreads);
    mbar_init(bar_drain, 1);
    *s_err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int wlim = a.wait_limit > 0 ? a.wait_limit : kWaitPolls;
  const int ntiles = (a.ncells + kInferRows - 1) / kInferRows;
  auto k_of = [&](int l) { return l == 0 ? a.in_pad : a.hidden; };
  auto n_of = [&](int ni, int l) { return l == a.nlin - 1 ? a.net[ni].out_pad : a.hidden; };

  if (warp == kProdWarp) {
    // ---- weight producer: every chunk of every step, in step order, into the ring
    if (lane == 0) {
      int gc = 0;
      bool bad = false;
      for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x)
        for (int ni = 0; ni < a.nnets && !bad; ++ni)
          for (int l = 0; l < a.nlin && !bad; ++l) {
            const int K = k_of(l), N = n_of(ni, l);
            for (int c = 0; c * kWChunkK < K; ++c, ++gc) {
              const int s = gc % kWStages;
              const uint32_t use = (uint32_t)(gc / kWStages);
              // the stage's previous chunk must have been consumed by its MMAs
              if (use > 0 && !mbar_wait(&bar_free[s], (use - 1) & 1, wlim, s_err)) {
                bad = true;
                break;
              }
              const int kc = min(kWChunkK, K - c * kWChunkK);
              const uint32_t bytes = (uint32_t)N * kc * 2;
              mbar_expect_tx(&bar_full[s], bytes);
              bulk_g2s(sW + s * kSmemStage, a.net[ni].wpack + a.net[ni].w_off[l] + (long long)c * N * kWChunkK, bytes,
                       &bar_full[s]);
            }
          }
      if (bad) *s_err = 1;
      // drain: every issued copy lands before the CTA exits (the last use of each stage)
      for (int s = 0; s < kWStages && s < gc; ++s) {
        const int last = gc - 1 - ((gc - 1 - s) % kWStages);
        if (!mbar_wait(&bar_full[s], (uint32_t)(last / kWStages) & 1)) *s_err = 1;
      }
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    // ---- MMA issuer
    if (lane == 0) {
      int gc = 0, step = 0;
      bool bad = false;
      const uint32_t abase = smem_u32(sA);
      for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x)
        for (int ni = 0; ni < a.nnets && !bad; ++ni)
          for (int l = 0; l < a.nlin && !bad; ++l, ++step) {
            const int K = k_of(l), N = n_of(ni, l);
            // the step's A operand is written and the accumulator has been read out
            if (!mbar_wait(bar_ain, (uint32_t)step & 1, wlim, s_err)) {
              bad = true;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t idesc = umma_idesc(kInferRows, N);
            const uint32_t a_sbo = (uint32_t)K * 16;
            for (int c = 0; c * kWChunkK < K; ++c, ++gc) {
              const int s = gc % kWStages;
              if (!mbar_wait(&bar_full[s], (uint32_t)(gc / kWStages) & 1, wlim, s_err)) {
                bad = true;
                break;
              }
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              const int kc = min(kWChunkK, K - c * kWChunkK);
              const uint32_t wbase = smem_u32(sW + s * kSmemStage);
              for (int kk = 0; kk < kc; kk += 16) {
                const int kg = c * kWChunkK + kk;
                const uint64_t ad = umma_desc(abase + (uint32_t)(kg >> 3) * 128, 128, a_sbo);
                const uint64_t bd = umma_desc(wbase + (uint32_t)(kk >> 3) * 128, 128, (uint32_t)kc * 16);
                umma_bf16(tmem, ad, bd, idesc, (c > 0 || kk > 0) ? 1u : 0u);
              }
              umma_commit(&bar_free[s]);
            }
            // test hook: the first step's completion signal withheld (its MMAs run and drain)
            if (!bad && !(a.fault == 1 && step == 0)) umma_commit(bar_acc);
          }
      if (bad) *s_err = 1;
      // drain: every issued MMA completes before the tensor memory is freed
      umma_commit(bar_drain);
      if (!mbar_wait(bar_drain, 0)) *s_err = 1;
    }
    __syncwarp();
  } else {
    // ---- features and epilogue: the two threads of a cell are lanes 2r and 2r + 1 of one warp
    const int row = tid >> 1, part = tid & 1;
    const int half = (a.ns + 1) >> 1, k0 = part * half, kn = min(half, a.ns - k0);
    __nv_bfloat162 fsp[kFeatSpecies];
    __nv_bfloat162 fx0 = __floats2bfloat162_rn(0.f, 0.f), fx1 = fx0;
    // column of species k's log feature (k != bath); its linear feature is ns columns further
    auto log_col = [&](int k) { return 2 + (k < a.bath ? k : k - 1); };
    // this thread's share of the tile's inputs, normalised, packed as BF16: species k0 + j as
    // (log10 Y, Y) pairs; thread part 0 also holds T, log P and log10 dt
    auto features = [&](int tile) {
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
      const double other = __shfl_xor_sync(0xffffffffu, ps, 1);
      const double rho = live ? (part == 0 ? ps + other : other + ps) : 1.0;
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
      float f0 = 0.f, f1 = 0.f, f2 = 0.f;
      if (live && part == 0) {
        f0 = ((float)(xT / rho) - a.fmean[0]) * a.fistd[0];
        f1 = ((float)a.logp - a.fmean[1]) * a.fistd[1];
        f2 = ((float)log10(fmax(dt, 1e-30)) - a.fmean[a.ns + 1]) * a.fistd[a.ns + 1];
      }
      fx0 = __floats2bfloat162_rn(f0, f1);
      fx1 = __floats2bfloat162_rn(f2, 0.f);
    };
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
    // hand the A operand to the MMA issuer: the generic-proxy writes are made visible to the
    // tensor core, and this thread's tensor-memory reads are ordered before the signal
    auto signal_a = [&]() {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(bar_ain);
    };
    if (blockIdx.x < ntiles) {
      features(blockIdx.x);
      write_inputs();
      signal_a();
    }
    const int erow = (warp & 3) * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    int step = 0;
    bool bad = false;
    for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x)
      for (int ni = 0; ni < a.nnets && !bad; ++ni)
        for (int l = 0; l < a.nlin && !bad; ++l, ++step) {
          const InferNet& net = a.net[ni];
          const int N = n_of(ni, l);
          // one lane per warp polls the accumulator barrier, the warp follows
          bool ok = true;
          if (lane == 0) ok = mbar_wait(bar_acc, (uint32_t)step & 1, wlim, s_err);
          ok = __shfl_sync(0xffffffffu, ok, 0);
          if (!ok) {
            bad = true;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          // warps w and w + 4 read the same TMEM lane quarter (rows), alternate 32-column groups
          const float* bl = net.bias + net.b_off[l];
          const bool last = l == a.nlin - 1;
          const int cell = tile * kInferRows + erow;
          for (int c0 = (warp >> 2) * 32; c0 < N; c0 += 64) {
            float v[32];
            tmem_ld32(trow + (uint32_t)c0, v);
            const int nc = min(32, N - c0);
            if (last) {
              if (cell < a.ncells) {
                float* o = net.out + (long long)cell * net.out_pad + c0;
#pragma unroll
                for (int i = 0; i < 32; ++i)
                  if (i < nc) o[i] = v[i] + __ldg(bl + c0 + i);
              }
            } else {
              // bias and GELU on pairs of columns (packed FP32), packed to BF16 pairs
              const float4* b4 = reinterpret_cast<const float4*>(bl + c0);
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const float4 ba = __ldg(b4 + 2 * q), bb = __ldg(b4 + 2 * q + 1);
                const f32x2 bp[4] = {f2_pack(ba.x, ba.y), f2_pack(ba.z, ba.w), f2_pack(bb.x, bb.y), f2_pack(bb.z, bb.w)};
                uint32_t w[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                  const f32x2 g = gelu2(f2_add(f2_pack(v[q * 8 + 2 * i], v[q * 8 + 2 * i + 1]), bp[i]));
                  const __nv_bfloat162 pb = __floats2bfloat162_rn(f2_lo(g), f2_hi(g));
                  w[i] = *reinterpret_cast<const uint32_t*>(&pb);
                }
                *reinterpret_cast<uint4*>(sA + canon_off(erow, c0 + q * 8, a.hidden)) = make_uint4(w[0], w[1], w[2], w[3]);
              }
            }
          }
          // the next step's A operand: the next layer's input is written above; after a
          // network's last layer (which writes only the outputs, so nothing else touches A) the
          // next network's inputs, or the next tile's features. The MMA issuer starts the next
          // step once all 256 threads have signalled, i.e. have also finished reading TMEM.
          if (last) {
            if (ni + 1 < a.nnets) {
              write_inputs();
            } else if (tile + (int)gridDim.x < ntiles) {
              features(tile + (int)gridDim.x);
              write_inputs();
            } else {
              continue;  // the CTA's last step: nothing follows
            }
          }
          signal_a();
        }
    if (bad) *s_err = 1;
  }
  // all roles finished (after an error every role stops at its next wait and drains its own work)
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (tid == 0 && *s_err && a.error) atomicExch(a.error, 1);
  if (warp == kMmaWarp) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem));
}

}  // namespace tng
