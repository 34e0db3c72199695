// K3: the implicit chemistry substep on sm_100a, one cell per warp.
//
// Replaces finitechem_source_chemistry's per-cell CVODE call (combustion/finitechem.f90:
// 962-1071): variable-order (1..5), variable-step BDF in Nordsieck form with modified Newton on
// M = I - gamma J and a dense FP64 LU with partial pivoting, stopping exactly at dt. The
// algorithm is restated in oracle/solver_oracle.c (the CPU twin used by the tests).
//
// Execution model (B200):
//  * a warp owns one cell; every vector of length NV = N+1 lives in registers, two entries per
//    lane (index lane and lane+32), so predictor, corrector update and WRMS norms are register
//    work plus one warp reduction;
//  * the right-hand side is table-driven and lane-parallel over the mechanism's reaction slots
//    (rates W_r into shared memory), production rates gathered from balanced per-lane chunk
//    lists (no atomics: results are deterministic);
//  * the Jacobian is assembled in shared memory (analytic mass-action and third-body/falloff-[M]
//    columns, forward-difference temperature column, temperature row from the species rows);
//    M = I - gamma J is factored in place by the warp (shuffle arg-max pivoting, 4x8 lane tiles
//    for the trailing update);
//  * a persistent grid steals cells from a queue; a cell that exhausts the pass's step budget
//    saves its Nordsieck history and goes to the next pass's queue (recompaction), so a pass
//    never runs longer than the budget allows and the host loop over passes is a CUDA graph;
//  * at eight warps per SM (two per scheduler) the kernel is bound by instruction supply and
//    latency, not by a pipe: the tables' records have odd strides (conflict-free lane-parallel
//    reads), the exponential's precision is fixed per kernel (one form in its code), the walks
//    are software-pipelined, transcendentals and the step control's divisions are out of line
//    except the plain-slot exponential, and the step control skips work whose outcome its
//    operands already decide. Each of these was kept on a measured, bit-identical A/B.
// No wait in this kernel depends on another warp or block: work is claimed with atomics only.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "solver_layout.h"
#include "tng_device.cuh"

namespace tng {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kQmax = 5;

// The solver tables of a handle as the host passes them: device pointers, the layout, precision.
struct SvDev {
  const double* __restrict__ hd;  // hot doubles
  const int* __restrict__ hi;     // hot ints
  const int* __restrict__ ci;     // cold ints
  SvLayout L;
  int mixed;  // rate-constant exponentials on the FP32 special-function unit (selects the kernels)
};

// A mechanism's layout with the precision of the rate-constant exponentials (kMixed: 0 FP64, 1 the
// mixed form) as a compile-time constant: the solver's kernels are instantiated on SvLX<LY, 0> and
// SvLX<LY, 1>, and the host picks by the handle's precision.
template <class LY, int MIX>
struct SvLX : LY {
  static constexpr int kMixed = MIX;
};

// Table view inside a kernel, specialised on the mechanism's layout LY (generated SvL_<m>: the
// sizes and table offsets are compile-time constants, so a table access is one shared-memory
// load at a fixed offset and every loop bound is known): hot tables in shared memory (staged per
// block), cold tables in shared memory when they fit, else global (read through L1).
template <class LY>
struct SvT {
  static constexpr int NS = LY::size(SZ_NS), NV = LY::size(SZ_NV), NSLOT = LY::size(SZ_NSLOT);
  static constexpr int NM = LY::size(SZ_NM), NFC = LY::size(SZ_NFC), NCD = LY::size(SZ_NCDCHUNK);
  static constexpr int NGP = LY::size(SZ_NGPAIR), NFO = LY::size(SZ_NFO);
  static constexpr int NCDSTEP = LY::size(SZ_NCDSTEP), NJDSTEP = LY::size(SZ_NJDSTEP);
  static constexpr int RS = (NV % 2 == 0) ? NV + 1 : NV;  // matrix row stride (odd: fewer bank conflicts)
  const double* __restrict__ hd;
  const int* __restrict__ hi;
  const int* __restrict__ ci;
  __device__ __forceinline__ const double* d(int k) const { return hd + LY::hd(k); }
  __device__ __forceinline__ const int* i(int k) const { return hi + LY::hi(k); }
  __device__ __forceinline__ const int* c(int k) const { return ci + LY::ci(k); }
};

__host__ __device__ inline int hot_smem_bytes(const SvLayout& L) { return L.nhd * 8 + L.nhi * 4; }
__host__ __device__ inline int cold_smem_doubles(const SvLayout& L) { return (L.nci * 4 + 15) / 16 * 2; }

// Copy the hot tables from global memory into the block's shared memory (all threads).
template <class LY>
__device__ __forceinline__ SvT<LY> stage_tables(const SvDev& g, void* smem) {
  double* d = reinterpret_cast<double*>(smem);
  int* i = reinterpret_cast<int*>(d + LY::nhd);
  const double2* gs = reinterpret_cast<const double2*>(g.hd);
  double2* ds = reinterpret_cast<double2*>(d);
  for (int e = threadIdx.x; e < LY::nhd / 2; e += blockDim.x) ds[e] = gs[e];
  const int4* gi = reinterpret_cast<const int4*>(g.hi);
  int4* di = reinterpret_cast<int4*>(i);
  for (int e = threadIdx.x; e < LY::nhi / 4; e += blockDim.x) di[e] = gi[e];
  __syncthreads();
  SvT<LY> t;
  t.hd = d;
  t.hi = i;
  t.ci = g.ci;
  return t;
}

// Copy the cold tables (the Jacobian's term lists) into shared memory at `at` (all threads),
// when the block has room for them; otherwise they are read from global memory through L1,
// which the shared-memory carve-out leaves small.
template <class LY>
__device__ __forceinline__ SvT<LY> stage_cold_tables(SvT<LY> t, double* at) {
  int* d = reinterpret_cast<int*>(at);
  for (int e = threadIdx.x; e < LY::nci; e += blockDim.x) d[e] = t.ci[e];
  __syncthreads();
  t.ci = d;
  return t;
}

// status codes per cell
enum { ST_OK = 0, ST_MAXSTEPS = 1, ST_CONVFAIL = 2, ST_ERRFAIL = 3, ST_NONFINITE = 4, ST_HMIN = 5, ST_PENDING = 9 };

struct BdfArgs {
  SvDev tab;
  double* state;     // species-major [v*ld + cell], in/out
  long long ld;
  const double* dts;  // per-cell dt or null
  double dt_scalar;
  double p;
  const int* queue_in;  // cells of this pass (null: 0..n_in-1)
  int n_in;
  int* head;        // work-stealing counter
  int* queue_out;   // cells that did not finish within the budget
  int* n_out;
  double* save;     // per-cell saved integrator state (save_stride doubles per cell)
  int save_stride;
  int* resume;      // per cell: 1 = integrator state in save
  int budget;       // internal steps per cell and pass
  double rtol, atol, dgmax;
  int max_steps, maxcor, msbp;
  int* nst;         // per-cell counters (accumulated over passes)
  int* nni;
  int* nje;
  int* status;
  int smem_warp;    // doubles of shared memory per warp
  int rs;           // row stride of the matrix
};

// shared-memory regions of one warp (offsets in doubles)
struct WarpMem {
  double* mat;  // NV x rs
  double* W;    // nslot: rates (RHS) or rate constants (Jacobian), by processing position
  double* C;    // 64 concentrations
  double* Ms;   // nm third-body sums
  double* lcm;  // nm log concentration for falloff
  double* fc;   // nfc x 3 (ln Fc, Troe N, Troe C)
  double* part; // ncdchunk partial production rates
  double* G;    // ngpair
  double* vb;   // 64 vector buffer
  double* hb;   // 64 enthalpies
  double* cb;   // 64 heat capacities (Jacobian), then the pivot reciprocals of the LU
  double* pr;   // nfo: Pr of the falloff slots (from the rate pass the Jacobian follows)
  double* cp;   // 8: the cell's CellPrep from the last rate pass
  int* perm;    // 64: the composed row permutation of the LU
};

__host__ __device__ inline int warp_mem_doubles(const SvLayout& L, int rs) {
  const int nv = L.size[SZ_NV];
  return nv * rs + L.size[SZ_NSLOT] + 64 + 2 * L.size[SZ_NM] + 3 * L.size[SZ_NFC] + L.size[SZ_NCDCHUNK] +
         L.size[SZ_NGPAIR] + 3 * 64 + L.size[SZ_NFO] + 8 + 32 /* the permutation as ints */ + 8;
}

template <class LY>
__device__ __forceinline__ WarpMem warp_mem(double* base) {
  using T = SvT<LY>;
  WarpMem w;
  double* p = base;
  w.mat = p; p += T::NV * T::RS;
  w.W = p; p += T::NSLOT;
  w.C = p; p += 64;
  w.Ms = p; p += T::NM;
  w.lcm = p; p += T::NM;
  w.fc = p; p += 3 * T::NFC;
  w.part = p; p += T::NCD;
  w.G = p; p += T::NGP;
  w.vb = p; p += 64;
  w.hb = p; p += 64;
  w.cb = p; p += 64;
  w.pr = p; p += T::NFO;
  w.cp = p; p += 8;
  w.perm = reinterpret_cast<int*>(p);
  return w;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  return __shfl_sync(kFull, v, 0);
}

__device__ __forceinline__ double expo(const double lnA, const double E, const double n, const int fl, const double LT,
                                       const double invRT) {
  double e = lnA;
  if (fl & 4) e = fma(E, invRT, e);
  if (fl & 2) e = fma(n, LT, e);
  return e;
}

__device__ __forceinline__ int nu_of(const int term) { return (int)(int8_t)(term & 0xFF); }

// One out-of-line copy of each transcendental the solver evaluates: inlined at every call site,
// the FP64 exp / log sequences made up a third of the right-hand side's code, and the solver's
// warps stalled on instruction fetch.
static __device__ __noinline__ double exp_ool(const double x) { return exp(x); }
static __device__ __noinline__ double log_ool(const double x) { return log(x); }
// IEEE division out of line, for the integrator's step control: inlined, each of its two dozen
// divisions carried its own reciprocal sequence (the quotient is correctly rounded either way)
static __device__ __noinline__ double div_ool(const double a, const double b) { return a / b; }

// exp in mixed precision: 2^x split into an exact power of two (FP64 scaling) and a fraction in
// [0, 1) evaluated by the FP32 ex2 unit, relative error about 3e-7.
static __device__ __noinline__ double exp_mixed_ool(const double e) {
  const double x = e * 1.4426950408889634;
  const double n = floor(x);
  if (!(n > -1100.0)) return 0.0;
  return ldexp((double)tng_ex2f((float)(x - n)), (int)fmin(n, 1100.0));
}

// exp of a rate-constant exponent in the kernel's precision (FP64, or the mixed form above),
// fixed at compile time by the layout (SvLX): a kernel carries the code of one form only, which
// keeps the other out of its instruction cache. The exponent itself (ln A + n ln T - E/RT, where
// the reverse rates' cancellations sit) is always formed in FP64.
template <class LY>
__device__ __forceinline__ double rexp(const SvT<LY>&, const double e) {
  if constexpr (LY::kMixed)
    return exp_mixed_ool(e);
  else
    return exp_ool(e);
}

// Per-cell thermochemical state shared by the rate and Jacobian evaluations.
struct CellPrep {
  double rho, T, LT, invRT, invT, irho;
};

// Stage the state (two entries per lane) and fill C, third-body sums, falloff [M] logs and the
// F_cent terms in shared memory.
template <class LY>
__device__ __forceinline__ CellPrep prepare(const SvT<LY>& t, const WarpMem& w, const double y0, const double y1,
                                           const double p, const int lane) {
  constexpr int ns = SvT<LY>::NS, nv = ns + 1, nm = SvT<LY>::NM, nfc = SvT<LY>::NFC;
  const double* sc = t.d(HD_SCAL);
  const double* invw = t.d(HD_INVW);
  if (lane < nv) w.vb[lane] = y0;
  if (lane + 32 < nv) w.vb[lane + 32] = y1;
  CellPrep c;
  c.rho = warp_sum((lane < ns ? y0 : 0.0) + (lane + 32 < ns ? y1 : 0.0));
  __syncwarp();
  c.irho = 1.0 / c.rho;
  c.T = w.vb[ns] / c.rho;  // by division, as the reference (the T > 1000 range switch is strict)
  c.LT = log_ool(c.T);
  c.invRT = 1.0 / (sc[SC_RGAS] * c.T);
  c.invT = sc[SC_RGAS] * c.invRT;
  if (lane < ns) w.C[lane] = y0 * invw[lane];
  if (lane + 32 < ns) w.C[lane + 32] = y1 * invw[lane + 32];
  __syncwarp();
  const double prt = p * c.invRT;  // [M] of the ideal gas, for a third-body sum that is zero
  const double* eff = t.d(HD_EFF);
  // (the loops of the cell preparation stay rolled: fully unrolled they added 1.8 KB to the
  // right-hand side's 22.5 KB of code, and the rolled form measured faster)
  for (int m = lane; m < nm; m += 32) {
    const double* e = eff + m * eff_stride(ns);
    double acc = 0.0;
#pragma unroll 4
    for (int j = 0; j < ns; ++j) acc = fma(e[j], w.C[j], acc);
    w.Ms[m] = acc;
    w.lcm[m] = log_ool(acc > 0.0 ? acc : prt);
  }
  const int* fcf = t.i(HI_FC);
  const double* fcd = t.d(HD_FC);
  for (int f = lane; f < nfc; f += 32) {
    const int forms = fcf[f];
    double v = 0.0;
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
      const int form = (forms >> (4 * q)) & 15;
      if (form == 15) break;
      const double a = fcd[kFcRec * f + 2 * q], cc = fcd[kFcRec * f + 2 * q + 1];
      const double term = form == 2 ? a : a * exp_ool(form == 0 ? -c.T * cc : -cc * c.invT);
      v = q == 0 ? term : v + term;
    }
    const double lfc = log_ool(v);
    const double l10 = lfc * sc[SC_INVLN10];
    w.fc[3 * f] = lfc;
    w.fc[3 * f + 1] = sc[SC_TN0] - sc[SC_TN1] * l10;
    w.fc[3 * f + 2] = -sc[SC_TC0] - sc[SC_TC1] * l10;
  }
  __syncwarp();
  return c;
}

// Rate constant of a falloff slot from its falloff word w1 (GETLINDRATECOEFF-equivalent:
// Lindemann, or Troe in log form); also returns Pr.
template <class LY>
__device__ __forceinline__ double falloff_const(const SvT<LY>& t, const WarpMem& w, const CellPrep& c, const int w1,
                                               double* pr_out) {
  const int f = w1 >> 8;
  const double* par = t.d(HD_FO) + kFoRec * f;
  const int fw = t.i(HI_FO)[f];
  const double* sc = t.d(HD_SCAL);
  const double lk0 = expo(par[0], par[1], par[2], fw & 15, c.LT, c.invRT);
  const double lki = expo(par[3], par[4], par[5], (fw >> 4) & 15, c.LT, c.invRT);
  const double lpr = lk0 + w.lcm[fw >> 16] - fmax(lki, sc[SC_LNKMIN]);
  const double pr = rexp(t, lpr);
  *pr_out = pr;
  const int fid = ((fw >> 8) & 255) - 1;
  double lk = lki;  // Lindemann: k_inf Pr / (1 + Pr)
  if (fid >= 0) {   // Troe: k_inf F Pr / (1 + Pr), ln F = ln Fc / (1 + f^2)
    const double lg = lpr * sc[SC_INVLN10] + w.fc[3 * fid + 2];
    const double ff = lg / (w.fc[3 * fid + 1] - sc[SC_TD] * lg);
    lk = lki + w.fc[3 * fid] / (ff * ff + 1.0);
  }
  return rexp(t, lk) * pr / (1.0 + pr);
}

// Rate constant of a plain (Arrhenius or constant) slot: the table holds (ln A, E, n) with zeros
// for absent terms, so the FMA chain of expo() gives the same exponent; constant slots hold A
// itself. The constant slots come last in processing order, so the rounds of 32 slots that hold
// only constants skip the exponential (one round per mechanism mixes the two kinds). This loop
// evaluates most of the right-hand side's exponentials, and its FP64 exp is the one inlined copy
// (the call and the registers it keeps live measured 3.5 % of the solve).
template <class LY>
__device__ __forceinline__ double plain_const(const SvT<LY>& t, const CellPrep& c, const int p, const int w0) {
  const double* sd = t.d(HD_SLOT) + kSlotRec * (p - SvT<LY>::NFO);
  const double a = sd[0];
  if (w0 & 8) return a;
  const double e = fma(sd[2], c.LT, fma(sd[1], c.invRT, a));
  if constexpr (LY::kMixed)
    return rexp(t, e);
  else
    return exp(e);
}

// The cell preparation and the slot loops of the right-hand side, one out-of-line copy (the
// solver's code must fit the instruction cache): W[q] = the slot's rate (its rate constant times
// the reactant concentrations and the third-body sum). With keep, the rate constants are also
// left in the matrix area (mat[q]) with Pr of the falloff slots (mat[NSLOT + q]), for the
// Jacobian formed next at the same state. The cell's CellPrep is left in w.cp.
template <class LY>
static __device__ __noinline__ void prep_rates(const SvT<LY> t, double* wb, const double y0, const double y1,
                                               const double p, const int lane, const int keep) {
  static_assert(SvT<LY>::NV * SvT<LY>::RS >= SvT<LY>::NSLOT + SvT<LY>::NFO, "kept constants fit the matrix area");
  const WarpMem w = warp_mem<LY>(wb);
  const CellPrep c = prepare(t, w, y0, y1, p, lane);
  static_assert(LY::hi(HI_SLOT) % 2 == 0, "slot words are read as int2");
  const int2* sw = reinterpret_cast<const int2*>(t.i(HI_SLOT));  // (w0, w1) per slot, one 8-byte read
  auto mass_action = [&](double v, const int w0, const int w1) {
    const int r0 = (w0 >> 4) & 127, r1 = (w0 >> 11) & 127, r2 = (w0 >> 18) & 127, mw = w1 & 127;
    if (r0 != kNone7) v = v * w.C[r0];
    if (r1 != kNone7) v = v * w.C[r1];
    if (r2 != kNone7) v = v * w.C[r2];
    if (mw != kNone7) v = v * w.Ms[mw];
    return v;
  };
  // the falloff slots (processing positions 0 .. NFO-1), then the plain and constant slots (one
  // round per mechanism mixes the two kinds; the others take one path). These loops, whose
  // bodies are large, stay rolled: unrolled or software-pipelined copies of them measured slower
  // (the code the eight warps of an SM share grows); only the small walks gained from it
  for (int q = lane; q < SvT<LY>::NFO; q += 32) {
    const int2 sq = sw[q];
    const int w0 = sq.x, w1 = sq.y;
    double pr = 0.0;
    const double k = falloff_const(t, w, c, w1, &pr);
    w.W[q] = mass_action(k, w0, w1);
    if (keep) {
      w.mat[q] = k;
      w.mat[SvT<LY>::NSLOT + q] = pr;
    }
  }
#pragma unroll 1
  for (int q = SvT<LY>::NFO + lane; q < SvT<LY>::NSLOT; q += 32) {
    const int2 sq = sw[q];
    const int w0 = sq.x, w1 = sq.y;
    const double k = plain_const(t, c, q, w0);
    w.W[q] = mass_action(k, w0, w1);
    if (keep) w.mat[q] = k;
  }
  if (lane == 0) {
    w.cp[0] = c.rho, w.cp[1] = c.T, w.cp[2] = c.LT, w.cp[3] = c.invRT, w.cp[4] = c.invT, w.cp[5] = c.irho;
  }
  __syncwarp();
}

__device__ __forceinline__ CellPrep load_prep(const WarpMem& w) {
  CellPrep c;
  c.rho = w.cp[0], c.T = w.cp[1], c.LT = w.cp[2], c.invRT = w.cp[3], c.invT = w.cp[4], c.irho = w.cp[5];
  return c;
}

// finitechem_compute_rhs for one cell, warp-cooperative. Input/output two entries per lane.
template <class LY>
__device__ __forceinline__ void rhs_warp(const SvT<LY>& t, const WarpMem& w, const double y0, const double y1,
                                         const double p, double& f0, double& f1, const int lane, const int keep) {
  constexpr int ns = SvT<LY>::NS;
  prep_rates<LY>(t, w.mat, y0, y1, p, lane, keep);
  const CellPrep c = load_prep(w);
  {
    // production-rate chunks: every lane walks the same number of steps over its interleaved
    // terms (conflict-free term reads, compile-time trip count) and stores a chunk's sum at the
    // chunk's last term. The walk is software-pipelined: the term of step st+2 and the rate of
    // step st+1 are requested before step st's arithmetic, so that a step waits on neither of
    // its two dependent shared-memory reads (with two warps per scheduler the walk is bound by
    // that latency, not by issue). The loop is unrolled by four, so that the integer and predicate
    // work of consecutive steps interleaves (by two measured 2 % faster than rolled, by four 0.7 %
    // more; the same unrolling of the Jacobian's walk was slower). The chunk sums go to a region
    // the walk never reads.
    constexpr int nst = SvT<LY>::NCDSTEP;
    if constexpr (nst > 0) {
      const int* __restrict__ ct = t.i(HI_CD_IL) + lane;
      const double* __restrict__ Wr = w.W;
      double* __restrict__ part = w.part;
      double acc = 0.0;
      int term = ct[0];
      double wv = Wr[(term >> 8) & 4095];
      int tn = nst > 1 ? ct[32] : 0;
#pragma unroll 4
      for (int st = 0; st < nst; ++st) {
        const double wn = Wr[(tn >> 8) & 4095];
        const int tnn = st + 2 < nst ? ct[32 * (st + 2)] : 0;
        if (term & 0xFF) acc = fma((double)nu_of(term), wv, acc);  // nu = 0: a padding step
        if (term & (1 << 20)) {
          part[(unsigned)term >> 21] = acc;
          acc = 0.0;
        }
        term = tn, wv = wn, tn = tnn;
      }
    }
  }
  __syncwarp();
  const int* spp = t.i(HI_CD_SP_PTR);
  const double* wm = t.d(HD_WMOL);
  const double* sc = t.d(HD_SCAL);
  const int toff = c.T > sc[SC_TMID] ? 0 : 12;
  const double* th = t.d(HD_TH);
  double cpm = 0.0, tmp = 0.0, r0 = 0.0, r1 = 0.0;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    const int k = lane + 32 * half;
    if (k < ns) {
      double cd = 0.0;
      for (int q = spp[k]; q < spp[k + 1]; ++q) cd += w.part[q];
      const double* a = th + kThStride * k + toff;
      const double T = c.T;
      const double cpk = a[0] * (a[7] + T * (a[8] + T * (a[9] + T * (a[10] + T * a[11]))));
      const double hk = a[0] * (T * (a[1] + T * (a[2] + T * (a[3] + T * (a[4] + T * a[5])))) + a[6]);
      const double rk = cd * wm[k];
      const double y = w.C[k] * (wm[k] * c.irho);
      cpm = fma(y, cpk, cpm);
      tmp = fma(-hk, rk, tmp);
      if (half == 0) r0 = rk; else r1 = rk;
    }
  }
  cpm = warp_sum(cpm);
  tmp = warp_sum(tmp);
  const double rT = tmp / cpm;
  f0 = lane < ns ? r0 : (lane == ns ? rT : 0.0);
  f1 = lane + 32 < ns ? r1 : (lane + 32 == ns ? rT : 0.0);
  __syncwarp();
}

// One out-of-line copy of the right-hand side. The solver evaluates it from several places;
// inlined at each of them, the kernel's code outgrows the instruction cache and the warps stall
// on instruction fetch.
// (The workspace is passed as its base pointer and its regions are recomputed from the
// compile-time layout, so that no descriptor goes through the stack.)
template <class LY>
static __device__ __noinline__ double2 rhs_call(const SvT<LY> t, double* wb, const double y0, const double y1,
                                                const double p, const int lane, const int keep = 0) {
  const WarpMem w = warp_mem<LY>(wb);
  double f0, f1;
  rhs_warp(t, w, y0, y1, p, f0, f1, lane, keep);
  return make_double2(f0, f1);
}

// Jacobian of the right-hand side at y (f = rhs(y) given), assembled into w.mat (row-major,
// row stride rs). Uses one extra right-hand side for the temperature column. It must follow the
// right-hand side at y evaluated with keep: the rate constants, Pr, concentrations, third-body
// sums and cell preparation are that evaluation's (the same values a new evaluation would give).
template <class LY>
__device__ __forceinline__ void jac_warp(const SvT<LY>& t, const WarpMem& w, const double y0, const double y1,
                                         const double f0, const double f1, const double p, const int lane) {
  constexpr int ns = SvT<LY>::NS, nv = ns + 1, rs = SvT<LY>::RS;
  for (int q = lane; q < SvT<LY>::NSLOT; q += 32) w.W[q] = w.mat[q];
  for (int q = lane; q < SvT<LY>::NFO; q += 32) w.pr[q] = w.mat[SvT<LY>::NSLOT + q];
  __syncwarp();
  const CellPrep c = load_prep(w);
  const int2* sw = reinterpret_cast<const int2*>(t.i(HI_SLOT));
#pragma unroll 1
  for (int e = lane; e < nv * rs; e += 32) w.mat[e] = 0.0;
  __syncwarp();
  // direct mass-action part: nu dW_p/dC_j for every reactant occurrence, the terms of one matrix
  // entry summed by one lane; the terms are interleaved by lane with the other reactants decoded
  // at generation time, so a step is one 8-byte term read and up to four independent loads.
  // Software-pipelined like the production-rate walk: the operands of step st+1 and the term of
  // step st+2 are requested before step st's arithmetic. An absent factor is read as 1.0 (a
  // product with 1.0 is exact, so the value is that of the skipped multiplication).
  constexpr int njs = SvT<LY>::NJDSTEP;
  if constexpr (njs > 0) {
    // (the matrix region never overlaps the slot, concentration and third-body regions read here)
    const int2* __restrict__ jt = reinterpret_cast<const int2*>(t.c(CI_JD_IL)) + lane;
    const double* __restrict__ Wr = w.W;
    const double* __restrict__ Cr = w.C;
    const double* __restrict__ Mr = w.Ms;
    double* __restrict__ mat = w.mat;
    const int2 pad = make_int2(kNone7 << 10 | kNone7 << 17 | kNone7 << 24, 0);
    auto operands = [&](const int2 tm, double& wv, double& ca, double& cb, double& mm) {
      const int pa = tm.x & 1023, ra = (tm.x >> 10) & 127, rb = (tm.x >> 17) & 127, mw = (tm.x >> 24) & 127;
      wv = Wr[pa];
      ca = ra != kNone7 ? Cr[ra] : 1.0;
      cb = rb != kNone7 ? Cr[rb] : 1.0;
      mm = mw != kNone7 ? Mr[mw] : 1.0;
    };
    double acc = 0.0;
    int2 tm = jt[0];
    double wv, ca, cb, mm;
    operands(tm, wv, ca, cb, mm);
    int2 tn = njs > 1 ? jt[32] : pad;
#pragma unroll 1
    for (int st = 0; st < njs; ++st) {
      double wv1, ca1, cb1, mm1;
      operands(tn, wv1, ca1, cb1, mm1);
      const int2 tnn = st + 2 < njs ? jt[32 * (st + 2)] : pad;
      const double d = ((wv * ca) * cb) * mm;
      if (tm.y & 0xFF) acc = fma((double)nu_of(tm.y), d, acc);  // nu = 0: a padding step
      if (tm.y & (1 << 20)) {
        mat[(tm.y >> 8) & 4095] = acc;
        acc = 0.0;
      }
      tm = tn, tn = tnn;
      wv = wv1, ca = ca1, cb = cb1, mm = mm1;
    }
  }
  // third-body and falloff-[M] part: G[i][m] = sum_p nu_ip dW_p/dM_m
  {
    const int* lp = t.c(CI_G_LANE_PTR);
    const int* ll = t.c(CI_G_LANE_LIST);
    const int* gb = t.c(CI_G_BEG);
    const int* ge = t.c(CI_G_END);
    const int* gt = t.c(CI_G_TERM);
    for (int i = lp[lane]; i < lp[lane + 1]; ++i) {
      const int g = ll[i];
      double acc = 0.0;
      for (int q = gb[g]; q < ge[g]; ++q) {
        const int term = gt[q];
        const int pp = term >> 12, kind = (term >> 8) & 15;
        const int2 sq = sw[pp];
        const int w0 = sq.x, w1 = sq.y;
        double prodC = 1.0;
#pragma unroll
        for (int o = 0; o < 3; ++o) {
          const int r = (w0 >> (4 + 7 * o)) & 127;
          if (r != kNone7) prodC *= w.C[r];
        }
        double val = 0.0;
        if (kind == 0) {
          val = w.W[pp] * prodC;
        } else {
          const int fw = t.i(HI_FO)[w1 >> 8];
          const double Mf = w.Ms[fw >> 16];
          if (Mf > 0.0) {
            const double pr = w.pr[pp];  // from the rate pass
            const int mw = w1 & 127;
            val = w.W[pp] / (Mf * (1.0 + pr)) * prodC * (mw != kNone7 ? w.Ms[mw] : 1.0);
          }
        }
        acc = fma((double)nu_of(term), val, acc);
      }
      w.G[g] = acc;
    }
  }
  __syncwarp();
  {
    constexpr int ng = SvT<LY>::NGP;
    const int* gi = t.c(CI_G_I);
    const int* gm = t.c(CI_G_M);
    const double* eff = t.d(HD_EFF);
    // the pairs are sorted by row: each row's contributions are summed in a register and added
    // to the matrix once (no read-modify-write chain through shared memory per pair); the loop
    // stays rolled (fully unrolled over the pairs it was a sixth of the solver's code). One pass
    // over the pairs serves all columns: lane j takes column j and, when there are more than 32
    // species, column j + 32 with a second accumulator, so the pairs' loads and row tests are not
    // repeated for a second round of a few columns.
    if constexpr (ng > 0) {
      const int j0 = lane, j1 = lane + 32;
      const bool c0 = j0 < ns, c1 = j1 < ns;
      int cur = gi[0];
      double acc0 = 0.0, acc1 = 0.0;
#pragma unroll 4
      for (int g = 0; g < ng; ++g) {
        const int row = gi[g];
        if (row != cur) {
          if (c0) w.mat[cur * rs + j0] += acc0;
          if (c1) w.mat[cur * rs + j1] += acc1;
          acc0 = 0.0, acc1 = 0.0;
          cur = row;
        }
        const double gv = w.G[g];
        const double* e = eff + gm[g] * eff_stride(ns);
        if (c0) acc0 = fma(gv, e[j0], acc0);
        if (c1) acc1 = fma(gv, e[j1], acc1);
      }
      if (c0) w.mat[cur * rs + j0] += acc0;
      if (c1) w.mat[cur * rs + j1] += acc1;
    }
  }
  __syncwarp();
  // temperature column: forward difference (one right-hand side)
  const double T = c.T, rho = c.rho;
  const double yN = __shfl_sync(kFull, ns < 32 ? y0 : y1, ns & 31);
  const double dlt = 1.4901161193847656e-08 * fmax(fabs(yN), 1e-30);
  const double yNp = yN + dlt;
  const double idl = 1.0 / (yNp - yN);
  const double2 gg = rhs_call(t, w.mat, lane == ns ? yNp : y0, lane + 32 == ns ? yNp : y1, p, lane);
  const double g0 = gg.x, g1 = gg.y;
  if (lane < nv) w.mat[lane * rs + ns] = (g0 - f0) * idl;
  if (lane + 32 < nv) w.mat[(lane + 32) * rs + ns] = (g1 - f1) * idl;
  __syncwarp();
  // species columns
  const double* wm = t.d(HD_WMOL);
  const double* iw = t.d(HD_INVW);
#pragma unroll 1
  for (int e = lane; e < ns * ns; e += 32) {
    const int i = e / ns, j = e % ns;
    w.mat[i * rs + j] = w.mat[i * rs + j] * (wm[i] * iw[j]) - T * w.mat[i * rs + ns];
  }
  // temperature row
  const double* sc = t.d(HD_SCAL);
  const int toff = T > sc[SC_TMID] ? 0 : 12;
  const double* th = t.d(HD_TH);
  double cpm = 0.0, ydcp = 0.0, scp = 0.0;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    const int k = lane + 32 * half;
    if (k < ns) {
      const double* a = th + kThStride * k + toff;
      const double cpk = a[0] * (a[7] + T * (a[8] + T * (a[9] + T * (a[10] + T * a[11]))));
      const double hk = a[0] * (T * (a[1] + T * (a[2] + T * (a[3] + T * (a[4] + T * a[5])))) + a[6]);
      const double dcp = a[0] * (a[8] + T * (2.0 * a[9] + T * (3.0 * a[10] + T * (4.0 * a[11]))));
      const double y = (half == 0 ? y0 : y1) / rho;
      cpm += y * cpk;
      ydcp += y * dcp;
      scp += cpk * (half == 0 ? f0 : f1);
      w.hb[k] = hk;
      w.cb[k] = cpk;
    }
  }
  cpm = warp_sum(cpm);
  ydcp = warp_sum(ydcp);
  scp = warp_sum(scp);
  const double fT = __shfl_sync(kFull, ns < 32 ? f0 : f1, ns & 31);
  __syncwarp();
  const double dTdu = -T / rho;
  {
    // one pass over the species rows for all columns (lane j: column j, and column j + 32 when
    // there are more than 32 species), four independent chains per column
    const int j0 = lane, j1 = lane + 32;
    const bool c0 = j0 < ns, c1 = j1 < ns;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    int k = 0;
#pragma unroll 1
    for (; k + 3 < ns; k += 4) {
      const double h0 = w.hb[k], h1 = w.hb[k + 1], h2 = w.hb[k + 2], h3 = w.hb[k + 3];
      if (c0) {
        s0 = fma(h0, w.mat[k * rs + j0], s0);
        s1 = fma(h1, w.mat[(k + 1) * rs + j0], s1);
        s2 = fma(h2, w.mat[(k + 2) * rs + j0], s2);
        s3 = fma(h3, w.mat[(k + 3) * rs + j0], s3);
      }
      if (c1) {
        t0 = fma(h0, w.mat[k * rs + j1], t0);
        t1 = fma(h1, w.mat[(k + 1) * rs + j1], t1);
        t2 = fma(h2, w.mat[(k + 2) * rs + j1], t2);
        t3 = fma(h3, w.mat[(k + 3) * rs + j1], t3);
      }
    }
#pragma unroll
    for (; k < ns; ++k) {
      if (c0) s0 = fma(w.hb[k], w.mat[k * rs + j0], s0);
      if (c1) t0 = fma(w.hb[k], w.mat[k * rs + j1], t0);
    }
    const double sum0 = (s0 + s1) + (s2 + s3), sum1 = (t0 + t1) + (t2 + t3);
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      const int j = h == 0 ? j0 : j1;
      if (j < ns) {
        double s = h == 0 ? sum0 : sum1;
        s += dTdu * scp;
        const double dcpm = (w.cb[j] - cpm) / rho + dTdu * ydcp;
        w.mat[ns * rs + j] = -(s + fT * dcpm) / cpm;
      }
    }
  }
  __syncwarp();
}

// In-place LU with partial pivoting (first maximum) of the N x N matrix a (row stride RS), for
// the compile-time size N, as the solver runs it:
//  * the pivot is the exact first maximum of |a[i][k]|, found with three warp reductions on the
//    64-bit pattern of |a| (a non-negative double orders like its bit pattern; NaN counts as 0)
//    instead of five rounds of shuffles;
//  * each lane keeps the pivot-row entries of its columns in registers for the trailing update,
//    so an update is one load and one store (4 x 8 lane tiles, rows walked at run time);
//  * the composed row permutation ((P b)[i] = b[perm[i]]) is kept up to date at each row exchange
//    and the pivots' reciprocals (dinv) are stored as they are formed, so that a solve runs in
//    registers with no pass over the factors afterwards.
// Returns nonzero if a pivot is zero or not finite (the factors are then not used).
template <int N, int RS>
__device__ __forceinline__ int lu_warp_t(double* __restrict__ a, int* perm, double* dinv, const int lane) {
  constexpr int NC = (N + 7) / 8;  // columns of a lane (8 column groups)
  int sing = 0;
  const int lr = lane >> 3, lc = lane & 7;
  for (int i = lane; i < N; i += 32) perm[i] = i;
  __syncwarp();
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    unsigned long long key = 0ULL;
    int bi = N;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = k + lane + 32 * h;
      if (i < N) {
        const double v = fabs(a[i * RS + k]);
        const unsigned long long kk = (v == v) ? (unsigned long long)__double_as_longlong(v) : 0ULL;
        if (bi == N || kk > key) key = kk, bi = i;
      }
    }
    const unsigned khi = (unsigned)(key >> 32), klo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(kFull, bi < N ? khi : 0u);
    const unsigned mlo = __reduce_max_sync(kFull, (bi < N && khi == mhi) ? klo : 0u);
    bi = (int)__reduce_min_sync(kFull, (bi < N && khi == mhi && klo == mlo) ? (unsigned)bi : 0xffffffffu);
    if (bi >= N) bi = k;  // no row (cannot happen for k < N)
    if (bi != k) {
      if (lane == 0) {
        const int t = perm[k];
        perm[k] = perm[bi];
        perm[bi] = t;
      }
      for (int j = lane; j < N; j += 32) {
        const double tmp = a[k * RS + j];
        a[k * RS + j] = a[bi * RS + j];
        a[bi * RS + j] = tmp;
      }
    }
    __syncwarp();
    const double d = a[k * RS + k];
    if (d == 0.0 || !isfinite(d)) {
      sing = 1;
      continue;
    }
    const double rd = 1.0 / d;
    if (lane == 0) dinv[k] = rd;
    for (int i = k + 1 + lane; i < N; i += 32) a[i * RS + k] *= rd;
    double u[NC];
#pragma unroll
    for (int p = 0; p < NC; ++p) {
      const int j = k + 1 + lc + 8 * p;
      u[p] = j < N ? a[k * RS + j] : 0.0;
    }
    __syncwarp();
    for (int i = k + 1 + lr; i < N; i += 4) {
      const double l = a[i * RS + k];
#pragma unroll
      for (int p = 0; p < NC; ++p) {
        const int j = k + 1 + lc + 8 * p;
        if (j < N) a[i * RS + j] = fma(-l, u[p], a[i * RS + j]);
      }
    }
    __syncwarp();
  }
  return sing;
}

// Out-of-line Jacobian and factorisation (one copy each, as rhs_call).
template <class LY>
static __device__ __noinline__ void jac_call(const SvT<LY> t, double* wb, const double y0, const double y1,
                                             const double f0, const double f1, const double p, const int lane) {
  jac_warp<LY>(t, warp_mem<LY>(wb), y0, y1, f0, f1, p, lane);
}

template <class LY>
static __device__ __noinline__ int lu_call(double* wb, const int lane) {
  using T = SvT<LY>;
  const WarpMem w = warp_mem<LY>(wb);
  return lu_warp_t<T::NV, T::RS>(w.mat, w.perm, w.cb, lane);
}

// Solve (LU) x = b with b and x two entries per lane in registers: permutation by one gather,
// forward and backward substitution by shuffles (no shared-memory round trips per step). Each
// substitution runs in two parts, over the pivots held in b0 (k < 32) and in b1 (k >= 32): the
// rows a pivot updates are then known per part (in the forward pass the pivots k >= 32 touch
// only rows of b1, in the backward pass the pivots k < 32 only rows of b0), and no part pays
// for the other's predicated-off loads and FMAs. The loops are unrolled by two (the compiler
// interleaves two columns' loads and index work; measured faster than both the rolled loop and a
// hand-pipelined one). The arithmetic per entry is unchanged.
__device__ __forceinline__ void lu_solve_reg(const double* a, const int n, const int rs, const int* perm,
                                             const double* dinv, double* vb, double& x0, double& x1, const int lane) {
  const int i0 = lane, i1 = lane + 32;
  if (i0 < n) vb[i0] = x0;
  if (i1 < n) vb[i1] = x1;
  __syncwarp();
  double b0 = i0 < n ? vb[perm[i0]] : 0.0;
  double b1 = i1 < n ? vb[perm[i1]] : 0.0;
  __syncwarp();
  const int nlo = n - 1 < 32 ? n - 1 : 32;  // forward pivots held in b0
#pragma unroll 2
  for (int k = 0; k < nlo; ++k) {
    const double bk = __shfl_sync(kFull, b0, k);
    if (i0 > k && i0 < n) b0 = fma(-a[i0 * rs + k], bk, b0);
    if (i1 < n) b1 = fma(-a[i1 * rs + k], bk, b1);
  }
#pragma unroll 2
  for (int k = 32; k < n - 1; ++k) {
    const double bk = __shfl_sync(kFull, b1, k - 32);
    if (i1 > k && i1 < n) b1 = fma(-a[i1 * rs + k], bk, b1);
  }
#pragma unroll 2
  for (int k = n - 1; k >= 32; --k) {
    const double bk = __shfl_sync(kFull, b1, k - 32) * dinv[k];
    if (i1 == k) b1 = bk;
    if (i0 < n) b0 = fma(-a[i0 * rs + k], bk, b0);
    if (i1 < k) b1 = fma(-a[i1 * rs + k], bk, b1);
  }
#pragma unroll 2
  for (int k = (n - 1 < 31 ? n - 1 : 31); k >= 0; --k) {
    const double bk = __shfl_sync(kFull, b0, k) * dinv[k];
    if (i0 == k) b0 = bk;
    if (i0 < k) b0 = fma(-a[i0 * rs + k], bk, b0);
  }
  x0 = b0;
  x1 = b1;
}

}  // namespace tng
