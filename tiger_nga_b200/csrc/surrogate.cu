// The surrogate substep: features and targets from implicit-solver pairs, normalisation,
// training (mlp.cu), BF16 weight packing, tensor-core inference (mlp_infer.cuh), the FP64
// conservation/renormalisation post-processing with fallback flags, the implicit fallback solve
// and the held-out judge. C-ABI tng_surrogate_* and tng_substep_surrogate.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <thread>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mlp.h"
#include "mlp_infer.cuh"
#include "solver.cuh"
#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

constexpr int kMaxNs = 64;
constexpr int kMaxEl = 8;

struct SurPost {
  double* state;
  long long ld;
  int ncells;
  const double* dts;
  double dt_scalar;
  double logp;
  int ns, bath, n_in, n_out, out_pad, nel;
  const float* out;      // network outputs, normalised
  const double* tmean;   // target mean/std, n_out
  const double* tstd;
  const float* fmin;     // raw-feature training range, n_in
  const float* fmax;
  double margin, consist_tol, clip_tol;
  const double* E;   // nel x ns: element atoms per kg of species (a_ek / W_k)
  const double* th;  // ns x 24 NASA (hi 12, lo 12)
  double tmid;
  int post_mode;     // 0: T from the enthalpy balance; 1: T from the network, enthalpy in the projection
  int members;       // ensemble members; outputs of member i at out + i * member_stride
  long long member_stride;
  double ens_tol_K, ens_tol_Y;
  // the error gate: a network that predicts log10 of this prediction's error relative to the
  // bars (|dT|/T over 1e-2, max |dY| / max Y over 1e-3); cells above log10(gate_tol) fall back
  const float* gate_out;  // normalised gate outputs [cell][gate_pad], null: no gate
  int gate_pad;
  double gate_mean[2], gate_std[2];
  double gate_log_tol;
  int* fb_list;      // fallback cells
  int* fb_count;
  unsigned long long* cnt;  // [accepted, ood, consistency, clip, ensemble, gate]
  double* out_state;  // predict mode: every cell's post-processed state here (state untouched, no list)
  long long ld_out;
  int* reason_out;    // per cell, nullable
  double* ind_out;    // per cell kIndicators values, nullable
  int cell_base;      // added to the fallback list's entries (the cells' place in the whole batch)
};

// per-cell indicators of tng_surrogate_predict: consistency (K), ensemble T spread (K), ensemble
// Y spread, gate log10(predicted T error / bar), gate log10(predicted Y error / bar)
constexpr int kIndicators = 5;

__device__ __forceinline__ void nasa(const double* th, double tmid, int k, double T, double* h, double* cp) {
  const double* a = th + kThStride * k + (T > tmid ? 0 : 12);
  *cp = a[0] * (a[7] + T * (a[8] + T * (a[9] + T * (a[10] + T * a[11]))));
  *h = a[0] * (T * (a[1] + T * (a[2] + T * (a[3] + T * (a[4] + T * a[5])))) + a[6]);
}

// the enthalpy alone (the same expression as nasa's h)
__device__ __forceinline__ double nasa_h(const double* th, double tmid, int k, double T) {
  const double* a = th + kThStride * k + (T > tmid ? 0 : 12);
  return a[0] * (T * (a[1] + T * (a[2] + T * (a[3] + T * (a[4] + T * a[5])))) + a[6]);
}

// raw features of one cell (same formulas as the inference kernel's featurisation)
__device__ __forceinline__ int raw_features(const double* state, long long ld, int cell, int ns, int bath, double logp,
                                            double dt, float* f, double* rho_out, double* T_out) {
  double rho = 0.0;
  for (int k = 0; k < ns; ++k) rho += state[(long long)k * ld + cell];
  const double T = state[(long long)ns * ld + cell] / rho;
  const int n_in = 2 * ns + 1;
  const double irho = 1.0 / rho;
  for (int i = 0; i < n_in; ++i) f[i] = sur_raw_input(i, ns, bath, state, ld, cell, irho, T, logp, dt);
  *rho_out = rho;
  *T_out = T;
  return n_in;
}

__global__ void k_sur_features(const double* __restrict__ state, long long ld, int n, const double* __restrict__ dts,
                               double logp, int ns, int bath, int in_pad, float* __restrict__ X) {
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < n; cell += gridDim.x * blockDim.x) {
    float f[2 * kMaxNs + 2];
    double rho, T;
    const int nf = raw_features(state, ld, cell, ns, bath, logp, dts[cell], f, &rho, &T);
    for (int i = 0; i < in_pad; ++i) X[(size_t)cell * in_pad + i] = i < nf ? f[i] : 0.f;
  }
}

// targets (dT, dY_k) of a pair, FP64 then stored as float
__global__ void k_sur_targets(const double* __restrict__ s0, const double* __restrict__ s1, long long ld, int n,
                              int ns, int out_pad, float* __restrict__ Tt) {
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < n; cell += gridDim.x * blockDim.x) {
    double r0 = 0.0, r1 = 0.0;
    for (int k = 0; k < ns; ++k) {
      r0 += s0[(long long)k * ld + cell];
      r1 += s1[(long long)k * ld + cell];
    }
    float* t = Tt + (size_t)cell * out_pad;
    const double T0 = s0[(long long)ns * ld + cell] / r0;
    t[0] = (float)((s1[(long long)ns * ld + cell] / r1 - T0) / T0);  // relative: the accuracy criterion's unit
    for (int k = 0; k < ns; ++k)
      t[1 + k] = (float)(s1[(long long)k * ld + cell] / r1 - s0[(long long)k * ld + cell] / r0);
    for (int i = ns + 1; i < out_pad; ++i) t[i] = 0.f;
  }
}

// per-column FP64 sum, sum of squares, min, max over rows (one block per column, fixed order)
__global__ void k_colstats(const float* __restrict__ A, int rows, int ld, double* __restrict__ out) {
  __shared__ double s1[256], s2[256], mn[256], mx[256];
  const int c = blockIdx.x;
  double a = 0.0, b = 0.0, lo = 1e300, hi = -1e300;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const double v = A[(size_t)r * ld + c];
    a += v;
    b += v * v;
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  s1[threadIdx.x] = a, s2[threadIdx.x] = b, mn[threadIdx.x] = lo, mx[threadIdx.x] = hi;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (threadIdx.x < off) {
      s1[threadIdx.x] += s1[threadIdx.x + off];
      s2[threadIdx.x] += s2[threadIdx.x + off];
      mn[threadIdx.x] = fmin(mn[threadIdx.x], mn[threadIdx.x + off]);
      mx[threadIdx.x] = fmax(mx[threadIdx.x], mx[threadIdx.x + off]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[4 * c] = s1[0], out[4 * c + 1] = s2[0], out[4 * c + 2] = mn[0], out[4 * c + 3] = mx[0];
  }
}

// A[r][c] = (A[r][c] - mean[c]) * scale[c] for c < ncol, 0 beyond
__global__ void k_normalise(float* __restrict__ A, int rows, int ld, int ncol, const float* __restrict__ mean,
                            const float* __restrict__ scale) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)rows * ld;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % ld);
    A[e] = c < ncol ? (A[e] - mean[c]) * scale[c] : 0.f;
  }
}

// FP32 parameters -> BF16 chunked canonical K-major layout of the inference kernel
__global__ void k_pack_weights(const float* __restrict__ W, int fo, int fi, __nv_bfloat16* __restrict__ dst) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < fo * fi; e += gridDim.x * blockDim.x) {
    const int n = e / fi, k = e % fi;
    const int c = k / kWChunkK, kk = k % kWChunkK;
    const int kc = min(kWChunkK, fi - c * kWChunkK);
    const int off = c * fo * kWChunkK + (int)(((n >> 3) * (kc * 16) + (kk >> 3) * 128 + (n & 7) * 16 + (kk & 7) * 2) / 2);
    dst[off] = __float2bfloat16_rn(W[e]);
  }
}

__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// prediction -> state with conservation; fallback cells keep their state and are listed
constexpr int kPostNs = 48;  // species of a cell held by the post-processing thread

// The mass fractions of one cell read from the state in place (Y_k = state[k] / rho): the state is
// read-only until the cell's result is stored, and a warp's reads of one species are one
// coalesced, L1-resident segment, whereas a per-thread copy would live in local memory.
struct CellY {
  const double* s;  // &state[cell]
  long long ld;
  double irho;      // 1 / rho
  __device__ __forceinline__ double operator[](int k) const { return s[(long long)k * ld] * irho; }
};

// Column k of the constraint matrix: the nel element rows (atoms per kg, a_ek / W_k), then, when
// NC > nel, the enthalpy row h_k(Th) * hsc.
template <int NC>
__device__ __forceinline__ void constraint_col(const SurPost& a, int k, double Th, double hsc, double (&c)[NC]) {
#pragma unroll
  for (int e = 0; e < NC; ++e) {
    if (e < a.nel) {
      c[e] = a.E[e * a.ns + k];
    } else {
      c[e] = nasa_h(a.th, a.tmid, k, Th) * hsc;
    }
  }
}

// Smallest change of dY in the metric sum dY'^2/D_k that satisfies the NC linear constraints
// A dY = b (b = 0 for the element rows, hrhs for the enthalpy row), by the normal equations
// G = A D A^T, G lam = A dY - b (Cholesky; NC is a compile-time count, so G and its factor stay
// in registers). Species driven below zero are pinned at zero (dY = -Y0, weight 0) and the
// projection repeated over the rest (an active set), so clipping keeps the constraints. A
// constraint whose carriers are all pinned or absent (G_ee = 0) holds already when its residual
// is zero and is then left out; otherwise, or when the active set does not settle, the cell is
// rejected (returns false).
template <int NC>
__device__ bool project_t(const SurPost& a, const CellY& Y0, double* dY, float* D, double Th, double hsc,
                          double hrhs) {
  for (int pass = 0; pass < 8; ++pass) {
    double G[NC][NC], r[NC], sc[NC];
#pragma unroll
    for (int e = 0; e < NC; ++e) {
      r[e] = e < a.nel ? 0.0 : -hrhs;
      sc[e] = e < a.nel ? 0.0 : fabs(hrhs);
#pragma unroll
      for (int g = 0; g < NC; ++g) G[e][g] = 0.0;
    }
    for (int k = 0; k < a.ns; ++k) {
      double c[NC];
      constraint_col<NC>(a, k, Th, hsc, c);
#pragma unroll
      for (int e = 0; e < NC; ++e) {
        r[e] = fma(c[e], dY[k], r[e]);
        sc[e] += fabs(c[e]) * (Y0[k] + fabs(dY[k]));
        const double cd = c[e] * (double)D[k];
#pragma unroll
        for (int g = 0; g <= e; ++g) G[e][g] = fma(cd, c[g], G[e][g]);
      }
    }
    bool act[NC];
#pragma unroll
    for (int e = 0; e < NC; ++e) {
      act[e] = G[e][e] > 0.0;
      if (!act[e] && !(fabs(r[e]) <= 1e-13 * sc[e] + 1e-300)) return false;
    }
#pragma unroll
    for (int i = 0; i < NC; ++i) {
#pragma unroll
      for (int j = 0; j <= i; ++j) {
        if (!act[i] || !act[j]) {
          G[i][j] = (i == j) ? 1.0 : 0.0;
          continue;
        }
        double sg = G[i][j];
#pragma unroll
        for (int q = 0; q < j; ++q) sg -= G[i][q] * G[j][q];
        if (i == j) {
          if (!(sg > 1e-14 * G[i][i])) return false;  // dependent constraints
          G[i][i] = sqrt(sg);
        } else {
          G[i][j] = sg / G[j][j];
        }
      }
    }
    double lam[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) {
      double sg = act[i] ? r[i] : 0.0;
#pragma unroll
      for (int q = 0; q < i; ++q) sg -= G[i][q] * lam[q];
      lam[i] = sg / G[i][i];
    }
#pragma unroll
    for (int i = NC - 1; i >= 0; --i) {
      double sg = lam[i];
#pragma unroll
      for (int q = i + 1; q < NC; ++q) sg -= G[q][i] * lam[q];
      lam[i] = sg / G[i][i];
    }
    bool pinned = false;
    for (int k = 0; k < a.ns; ++k) {
      if (D[k] == 0.0f) continue;
      double c[NC];
      constraint_col<NC>(a, k, Th, hsc, c);
      double corr = 0.0;
#pragma unroll
      for (int e = 0; e < NC; ++e) corr = fma(c[e], lam[e], corr);
      dY[k] -= (double)D[k] * corr;
      if (Y0[k] + dY[k] < 0.0) {
        dY[k] = -Y0[k];
        D[k] = 0.0f;
        pinned = true;
      }
    }
    if (!pinned) return true;
  }
  return false;  // still pinning species after eight passes: leave the cell to the implicit solve
}

// the projection for the run-time constraint count nc = nel (+1 with the enthalpy row)
__device__ bool project(const SurPost& a, int nc, const CellY& Y0, double* dY, float* D, double Th, double hsc,
                        double hrhs) {
  switch (nc) {
    case 1: return project_t<1>(a, Y0, dY, D, Th, hsc, hrhs);
    case 2: return project_t<2>(a, Y0, dY, D, Th, hsc, hrhs);
    case 3: return project_t<3>(a, Y0, dY, D, Th, hsc, hrhs);
    case 4: return project_t<4>(a, Y0, dY, D, Th, hsc, hrhs);
    case 5: return project_t<5>(a, Y0, dY, D, Th, hsc, hrhs);
    case 6: return project_t<6>(a, Y0, dY, D, Th, hsc, hrhs);
    case 7: return project_t<7>(a, Y0, dY, D, Th, hsc, hrhs);
    default: return project_t<8>(a, Y0, dY, D, Th, hsc, hrhs);
  }
}

// mass fractions after the projection: max(Y0 + dY, 0) renormalised to sum 1
__device__ __forceinline__ double y_new(const CellY& Y0, const double* dY, int k, double inv_sum) {
  return fmax(Y0[k] + dY[k], 0.0) * inv_sum;
}

// temperature with sum Y_k h_k(T) = h0 (Newton from T), Y = y_new(...). Within one NASA range
// the mixture enthalpy and heat capacity are polynomials in T whose coefficients are the
// Y-weighted sums of the species' (c0 a_i, c0 b_i): they are formed once per range visited, so
// a Newton iteration is two Horner chains instead of a pass over the species.
__device__ double enthalpy_T(const SurPost& a, const CellY& Y0, const double* dY, double inv_sum, double h0,
                             double T) {
  double ch[6], cc[5];  // H(T) = T (ch0 + T (ch1 + ... + T ch4)) + ch5, Cp(T) = cc0 + T (cc1 + ... + T cc4)
  int range = -1;
  for (int it = 0; it < 12; ++it) {
    const int r = T > a.tmid ? 0 : 1;
    if (r != range) {
      range = r;
#pragma unroll
      for (int i = 0; i < 6; ++i) ch[i] = 0.0;
#pragma unroll
      for (int i = 0; i < 5; ++i) cc[i] = 0.0;
      for (int k = 0; k < a.ns; ++k) {
        const double* t = a.th + kThStride * k + 12 * r;
        const double w = y_new(Y0, dY, k, inv_sum) * t[0];
#pragma unroll
        for (int i = 0; i < 6; ++i) ch[i] = fma(w, t[1 + i], ch[i]);
#pragma unroll
        for (int i = 0; i < 5; ++i) cc[i] = fma(w, t[7 + i], cc[i]);
      }
    }
    const double hh = T * (ch[0] + T * (ch[1] + T * (ch[2] + T * (ch[3] + T * ch[4])))) + ch[5];
    const double cp = cc[0] + T * (cc[1] + T * (cc[2] + T * (cc[3] + T * cc[4])));
    const double step = (hh - h0) / cp;
    T -= step;
    if (fabs(step) < 1e-9 * T) break;
  }
  return T;
}

// prediction -> state with conservation; fallback cells keep their state and are listed
__global__ void __launch_bounds__(128) k_sur_post(const SurPost a) {
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < a.ncells; cell += gridDim.x * blockDim.x) {
    const double dt = a.dts ? a.dts[cell] : a.dt_scalar;
    double rho = 0.0;
    for (int k = 0; k < a.ns; ++k) rho += a.state[(long long)k * a.ld + cell];
    const double T0 = a.state[(long long)a.ns * a.ld + cell] / rho;
    const double irho0 = 1.0 / rho;
    int reason = 0;
    for (int i = 0; i < a.n_in && !reason; ++i) {
      const float f = sur_raw_input(i, a.ns, a.bath, a.state, a.ld, cell, irho0, T0, a.logp, dt);
      const float span = a.fmax[i] - a.fmin[i];
      if (f < a.fmin[i] - a.margin * span || f > a.fmax[i] + a.margin * span) reason = 1;
    }
    // dY in double, the projection weights D in float (the constraints hold exactly for any
    // weights, since the normal equations use the same D); Y0 is read from the state in place
    double dY[kPostNs];
    float D[kPostNs];
    const CellY Y0{a.state + cell, a.ld, 1.0 / rho};
    // the ensemble: mean prediction, and the spread of the members as an error indicator
    const float* o = a.out + (size_t)cell * a.out_pad;
    double rT = 0.0, tlo = 1e300, thi = -1e300, sY = 0.0;
    for (int i = 0; i < a.members; ++i) {
      const double v = (double)o[i * a.member_stride] * a.tstd[0] + a.tmean[0];
      rT += v;
      tlo = fmin(tlo, v), thi = fmax(thi, v);
    }
    const double Tnet = fmin(fmax(T0 * (1.0 + rT / a.members), 200.0), 6000.0);
    const double sT = T0 * (thi - tlo);
    double neg = 0.0, h0 = 0.0;  // negative mass fraction the network predicted (clip test)
    for (int k = 0; k < a.ns; ++k) {
      double m = 0.0, lo = 1e300, hi = -1e300;
      for (int i = 0; i < a.members; ++i) {
        const double v = (double)o[i * a.member_stride + 1 + k] * a.tstd[1 + k] + a.tmean[1 + k];
        m += v;
        lo = fmin(lo, v), hi = fmax(hi, v);
      }
      dY[k] = m / a.members;
      sY = fmax(sY, hi - lo);
      D[k] = (float)(fabs(Y0[k]) + fabs(Y0[k] + dY[k]) + 1e-12);
      if (Y0[k] + dY[k] < 0.0) neg -= Y0[k] + dY[k];
      h0 = fma(Y0[k], nasa_h(a.th, a.tmid, k, T0), h0);
    }
    // species the network drives below zero are pinned at zero before the first pass (the
    // projection would pin them one pass at a time otherwise)
    for (int k = 0; k < a.ns; ++k)
      if (Y0[k] + dY[k] < 0.0) dY[k] = -Y0[k], D[k] = 0.0f;
    // element conservation, then the temperature the conserved Y implies
    bool ok = project(a, a.nel, Y0, dY, D, 0.0, 0.0, 0.0);
    double sum = 0.0;
    for (int k = 0; k < a.ns; ++k) sum += fmax(Y0[k] + dY[k], 0.0);
    double inv_sum = 1.0 / sum;
    double T1 = enthalpy_T(a, Y0, dY, inv_sum, h0, Tnet);
    const double ind = fabs(T1 - Tnet);
    if (ok && a.post_mode == 1) {
      // keep the network's temperature: move Y (elements held) until h(Y, Tnet) = h0; the
      // enthalpy row is scaled by 1 / (cp T)
      double cpm = 0.0, hy = 0.0;
      for (int k = 0; k < a.ns; ++k) {
        double hk, cpk;
        nasa(a.th, a.tmid, k, Tnet, &hk, &cpk);
        cpm = fma(y_new(Y0, dY, k, inv_sum), cpk, cpm);
        hy = fma(hk, Y0[k], hy);
      }
      const double hsc = 1.0 / (cpm * Tnet);
      ok = project(a, a.nel + 1, Y0, dY, D, Tnet, hsc, (h0 - hy) * hsc);
      sum = 0.0;
      for (int k = 0; k < a.ns; ++k) sum += fmax(Y0[k] + dY[k], 0.0);
      inv_sum = 1.0 / sum;
      T1 = enthalpy_T(a, Y0, dY, inv_sum, h0, Tnet);  // one correction for the renormalisation
    }
    if (!reason && !(ind <= a.consist_tol)) reason = 2;
    if (!reason && !(neg <= a.clip_tol)) reason = 3;
    if (!reason && !(isfinite(T1) && ok)) reason = 2;
    if (!reason && !(sT <= a.ens_tol_K && sY <= a.ens_tol_Y)) reason = 4;
    double gT = -INFINITY, gY = -INFINITY;
    if (a.gate_out) {
      const float* go = a.gate_out + (size_t)cell * a.gate_pad;
      gT = (double)go[0] * a.gate_std[0] + a.gate_mean[0];
      gY = (double)go[1] * a.gate_std[1] + a.gate_mean[1];
      if (!reason && !(gT <= a.gate_log_tol && gY <= a.gate_log_tol)) reason = 5;
    }
    if (a.reason_out) a.reason_out[cell] = reason;
    if (a.ind_out) {
      double* io = a.ind_out + kIndicators * (size_t)cell;
      io[0] = ok ? ind : INFINITY;
      io[1] = sT;
      io[2] = sY;
      io[3] = gT;
      io[4] = gY;
    }
    if (a.out_state) {
      for (int k = 0; k < a.ns; ++k) a.out_state[(long long)k * a.ld_out + cell] = rho * y_new(Y0, dY, k, inv_sum);
      a.out_state[(long long)a.ns * a.ld_out + cell] = rho * T1;
    } else if (reason) {
      const int slot = atomicAdd(a.fb_count, 1);
      a.fb_list[slot] = a.cell_base + cell;
      atomicAdd(&a.cnt[reason], 1ULL);
    } else {
      for (int k = 0; k < a.ns; ++k) a.state[(long long)k * a.ld + cell] = rho * y_new(Y0, dY, k, inv_sum);
      a.state[(long long)a.ns * a.ld + cell] = rho * T1;
      atomicAdd(&a.cnt[0], 1ULL);
    }
  }
}

__global__ void k_gather_cells(const double* __restrict__ src, long long ld, int nv, const int* __restrict__ idx, int m,
                               double* __restrict__ dst, long long dst_ld, const double* __restrict__ dts, double dt,
                               double* __restrict__ dts_out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    for (int v = 0; v < nv; ++v) dst[(long long)v * dst_ld + j] = src[(long long)v * ld + idx[j]];
    dts_out[j] = dts ? dts[idx[j]] : dt;
  }
}

// The fallback cells listed by the post-processing (count on the device) into columns J, J+1, ...
// of the joint batch, whose first J columns hold the judged sample; n_out = J + count.
__global__ void k_gather_list(const double* __restrict__ src, long long ld, int nv, const int* __restrict__ list,
                              const int* __restrict__ count, int J, double* __restrict__ dst, long long dst_ld,
                              const double* __restrict__ dts, double dt, double* __restrict__ dts_out,
                              int* __restrict__ n_out) {
  const int n = *count;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int c = list[j];
    for (int v = 0; v < nv; ++v) dst[(long long)v * dst_ld + J + j] = src[(long long)v * ld + c];
    dts_out[J + j] = dts ? dts[c] : dt;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = J + n;
}

// the solved fallback cells back into the state
__global__ void k_scatter_list(double* __restrict__ dst, long long ld, int nv, const int* __restrict__ list,
                               const int* __restrict__ count, int J, const double* __restrict__ src, long long src_ld) {
  const int n = *count;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    for (int v = 0; v < nv; ++v) dst[(long long)v * ld + list[j]] = src[(long long)v * src_ld + J + j];
}

// Processing order of the joint batch (judged sample in columns 0..J-1, the *count fallback
// cells after it): the fallback cells first -- the ones the surrogate could not take, usually the
// stiffest -- so that the longest integrations start earliest and the tail is shorter.
__global__ void k_joint_order(int* __restrict__ a, const int* __restrict__ count, int J, long long cap) {
  const long long n = *count;
  const long long m = (J + n < cap) ? J + n : cap;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    a[i] = (int)(i < n ? J + i : i - n);
}

// surrogate(+fallback) result vs implicit result on the judged cells
__global__ void k_judge(const double* __restrict__ state, long long ld, int ns, const int* __restrict__ idx, int m,
                        const double* __restrict__ ref, long long ref_ld, double* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const int c = idx[j];
    double rs = 0.0, rr = 0.0, ymax = 0.0;
    for (int k = 0; k < ns; ++k) {
      rs += state[(long long)k * ld + c];
      rr += ref[(long long)k * ref_ld + j];
    }
    for (int k = 0; k < ns; ++k) ymax = fmax(ymax, ref[(long long)k * ref_ld + j] / rr);
    const double Ts = state[(long long)ns * ld + c] / rs, Tp = ref[(long long)ns * ref_ld + j] / rr;
    double dy = 0.0;
    for (int k = 0; k < ns; ++k)
      dy = fmax(dy, fabs(state[(long long)k * ld + c] / rs - ref[(long long)k * ref_ld + j] / rr));
    atomic_max_pos(&out[0], fabs(Ts - Tp) / Tp);
    atomic_max_pos(&out[1], dy / ymax);
  }
}

// Per-cell error of a post-processed prediction against the implicit result, relative to the
// accuracy bars: r[0] = (|T_s - T_p| / T_p) / 1e-2, r[1] = (max_k |Y_s,k - Y_p,k| / max_k Y_p,k) / 1e-3.
__global__ void k_sur_errors(const double* __restrict__ pred, long long ldp, const double* __restrict__ ref,
                             long long ldr, int n, int ns, float* __restrict__ r) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double rs = 0.0, rr = 0.0, ymax = 0.0, dy = 0.0;
    for (int k = 0; k < ns; ++k) {
      rs += pred[(long long)k * ldp + c];
      rr += ref[(long long)k * ldr + c];
    }
    const double irs = 1.0 / rs, irr = 1.0 / rr;
    for (int k = 0; k < ns; ++k) {
      const double yr = ref[(long long)k * ldr + c] * irr;
      ymax = fmax(ymax, yr);
      dy = fmax(dy, fabs(pred[(long long)k * ldp + c] * irs - yr));
    }
    const double Ts = pred[(long long)ns * ldp + c] * irs, Tp = ref[(long long)ns * ldr + c] * irr;
    r[2 * (size_t)c] = (float)(fabs(Ts - Tp) / Tp / 1e-2);
    r[2 * (size_t)c + 1] = (float)(dy / ymax / 1e-3);
  }
}

// gate targets: log10 of the errors relative to the bars, floored at 1e-4 (normalised later)
__global__ void k_gate_targets(const float* __restrict__ r, int n, int out_pad, float* __restrict__ T) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    float* t = T + (size_t)c * out_pad;
    t[0] = log10f(fmaxf(r[2 * (size_t)c], 1e-4f));
    t[1] = log10f(fmaxf(r[2 * (size_t)c + 1], 1e-4f));
    for (int i = 2; i < out_pad; ++i) t[i] = 0.f;
  }
}

}  // namespace tng

using namespace tng;

constexpr int kMaxMembers = 4;

struct tng_surrogate {
  tng_chem* h = nullptr;
  tng_surrogate_cfg cfg{};
  Mlp m;                         // member 0 (also the member of the single-network tools)
  Mlp mx[kMaxMembers - 1];       // members 1 ..
  int members = 1;
  Mlp& member(int i) { return i == 0 ? m : mx[i - 1]; }
  const Mlp& member(int i) const { return i == 0 ? m : mx[i - 1]; }
  int ns = 0, bath = 0, n_in = 0, n_out = 0, nel = 0;
  std::vector<double> fmean, fstd, fmin, fmax, tmean, tstd;  // host copies
  bool trained = false;
  // device
  float* d_fnorm = nullptr;  // fmean (in_pad), fistd (in_pad), fmin (in_pad), fmax (in_pad)
  double* d_tnorm = nullptr;  // tmean (out_pad), tstd (out_pad)
  double* d_E = nullptr;
  __nv_bfloat16* d_wpack[kMaxMembers] = {};
  long long w_off[kMaxLayers] = {};
  DevBuf out, fb, cnt, judge_state, judge_dts, judge_idx, work, joint;
  cudaEvent_t ev[5] = {};
  int calls = 0;
  int dbg_wait_limit = 0, dbg_fault = 0;  // test hook of the inference kernel's bounded waits
  // the error gate (a network of the same hidden shape, 2 outputs); absent until trained or loaded
  bool has_gate = false;
  Mlp gate;
  double gate_mean[2] = {0.0, 0.0}, gate_std[2] = {1.0, 1.0};
  double gate_tol = 0.25;  // fallback above this fraction of the bars (calibrated, saved with the model)
  __nv_bfloat16* d_gpack = nullptr;
  long long g_off[kMaxLayers] = {};
  DevBuf gout;
  // the host-pointer substep's upload in chunks: a copy stream and one event per chunk (+ start)
  static constexpr int kPipeChunks = 16;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t pev[kPipeChunks + 1] = {};
  // ... and its download: the state after the post-processing goes back during the fallback
  // solve, then only the solved fallback cells (pinned staging, grown as needed)
  cudaEvent_t ev_front = nullptr, ev_down = nullptr;
  double* h_comp = nullptr;
  int* h_list = nullptr;
  size_t h_cap = 0;  // cells
};

static int sur_upload_norm(tng_surrogate* s) {
  const int ip = s->m.in_pad, op = s->m.out_pad;
  std::vector<float> f(4 * ip, 0.f);
  for (int i = 0; i < s->n_in; ++i) {
    f[i] = (float)s->fmean[i];
    f[ip + i] = (float)(1.0 / s->fstd[i]);
    f[2 * ip + i] = (float)s->fmin[i];
    f[3 * ip + i] = (float)s->fmax[i];
  }
  std::vector<double> t(2 * op, 0.0);
  for (int i = 0; i < s->n_out; ++i) {
    t[i] = s->tmean[i];
    t[op + i] = s->tstd[i];
  }
  cudaMemcpy(s->d_fnorm, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice);
  cudaError_t e = cudaMemcpy(s->d_tnorm, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "surrogate normalisation");
}

static void pack_net(tng_surrogate* s, const Mlp& mi, __nv_bfloat16* dst, long long* w_off) {
  long long off = 0;
  for (int l = 0; l < mi.nlin; ++l) {
    w_off[l] = off;
    const int fo = mi.fan_out[l], fi = mi.fan_in[l];
    k_pack_weights<<<256, 256, 0, s->m.stream>>>(mi.params + mi.w_off[l], fo, fi, dst + off);
    off += (long long)fo * fi;
  }
}

static int sur_pack(tng_surrogate* s) {
  for (int i = 0; i < s->members; ++i) pack_net(s, s->member(i), s->d_wpack[i], s->w_off);
  if (s->has_gate) pack_net(s, s->gate, s->d_gpack, s->g_off);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "surrogate weight packing");
}

// One launch of the tensor-core inference over nmembers ensemble members starting at
// first_member (outputs at out + i * ncells * out_pad) and, with gate, the error gate (outputs in
// s->gout): the cells' features are formed once for all of them.
static int launch_infer(tng_chem* h, tng_surrogate* s, const double* dstate, int64_t ncells, int64_t dld,
                        const double* ddts, double dt, double p, int first_member, int nmembers, float* out, bool gate,
                        int* err, int64_t gate_off = 0) {
  gate = gate && s->has_gate;
  if (gate && !s->gout.reserve((size_t)(gate_off + ncells) * s->gate.out_pad * sizeof(float)))
    return set_error(TNG_ERR_CUDA, "surrogate gate output allocation failed");
  InferArgs ia{};
  ia.state = dstate;
  ia.ld = dld;
  ia.ncells = (int)ncells;
  ia.dts = ddts;
  ia.dt_scalar = dt;
  ia.logp = std::log(p);
  ia.ns = s->ns;
  ia.bath = s->bath;
  ia.n_in = s->n_in;
  ia.in_pad = s->m.in_pad;
  ia.hidden = s->m.hidden;
  ia.nlin = s->m.nlin;
  ia.fmean = s->d_fnorm;
  ia.fistd = s->d_fnorm + s->m.in_pad;
  auto add = [&](const Mlp& net, const __nv_bfloat16* wpack, const long long* w_off, float* o) {
    InferNet& n = ia.net[ia.nnets++];
    n.wpack = wpack;
    for (int l = 0; l < net.nlin; ++l) {
      n.w_off[l] = w_off[l];
      n.b_off[l] = (int)net.b_off[l];
    }
    n.bias = net.params;
    n.out_pad = net.out_pad;
    n.out = o;
  };
  if (nmembers + (gate ? 1 : 0) < 1 || nmembers + (gate ? 1 : 0) > kMaxNets)
    return set_error(TNG_ERR_ARG, "inference: 1..%d networks per launch", kMaxNets);
  for (int i = 0; i < nmembers; ++i)
    add(s->member(first_member + i), s->d_wpack[first_member + i], s->w_off, out + (size_t)i * ncells * s->m.out_pad);
  if (gate) add(s->gate, s->d_gpack, s->g_off, (float*)s->gout.ptr + gate_off * s->gate.out_pad);
  ia.error = err;
  ia.wait_limit = s->dbg_wait_limit;
  ia.fault = s->dbg_fault;
  cudaError_t e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
  if (e != cudaSuccess) return cuda_error(e, "inference shared memory");
  const int grid = (int)std::min<int64_t>(2 * h->sm_count, (ncells + kInferRows - 1) / kInferRows);
  k_mlp_infer<<<grid, kInferThreads, kInferSmem, h->stream>>>(ia);
  e = cudaGetLastError();
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "tensor-core inference");
}

namespace tng {
// arguments of the post-processing kernel common to the substep and the plain prediction
static SurPost post_args(tng_chem* h, tng_surrogate* s, double* state, int64_t ld, int64_t ncells, const double* dts,
                         double dt, double p) {
  SurPost pa{};
  pa.state = state;
  pa.ld = ld;
  pa.ncells = (int)ncells;
  pa.dts = dts;
  pa.dt_scalar = dt;
  pa.logp = std::log(p);
  pa.ns = s->ns;
  pa.bath = s->bath;
  pa.n_in = s->n_in;
  pa.n_out = s->n_out;
  pa.out_pad = s->m.out_pad;
  pa.nel = s->nel;
  pa.out = (const float*)s->out.ptr;
  pa.tmean = s->d_tnorm;
  pa.tstd = s->d_tnorm + s->m.out_pad;
  pa.fmin = s->d_fnorm + 2 * s->m.in_pad;
  pa.fmax = s->d_fnorm + 3 * s->m.in_pad;
  pa.margin = s->cfg.ood_margin;
  pa.consist_tol = s->cfg.consist_tol_K;
  pa.clip_tol = s->cfg.clip_tol;
  pa.post_mode = s->cfg.post_mode;
  pa.members = s->members;
  pa.member_stride = (long long)ncells * s->m.out_pad;
  pa.ens_tol_K = s->cfg.ens_tol_K;
  pa.ens_tol_Y = s->cfg.ens_tol_Y;
  pa.E = s->d_E;
  solver_thermo(h, &pa.th, &pa.tmid);
  if (s->has_gate) {
    pa.gate_out = (const float*)s->gout.ptr;
    pa.gate_pad = s->gate.out_pad;
    for (int i = 0; i < 2; ++i) pa.gate_mean[i] = s->gate_mean[i], pa.gate_std[i] = s->gate_std[i];
    const double tol = s->cfg.gate_tol > 0.f ? (double)s->cfg.gate_tol : s->gate_tol;
    pa.gate_log_tol = std::log10(tol);
  }
  return pa;
}

// The front of the surrogate substep with host pointers, overlapped with the state's upload: the
// state (and per-cell dt) go to the device in chunks on the surrogate's copy stream, and on the
// handle's stream each chunk's judged cells are gathered and its cells inferred and
// post-processed as soon as its copy has landed. The judged cells (jidx on the device, ascending:
// joff + j * jstride) are gathered into jdst / jdts (leading dimension jld). ev[0] .. ev[1] bracket
// the interleaved front (ev[2] = ev[1]).
static int sur_front_pipelined(tng_chem* h, tng_surrogate* s, const double* state, int64_t ld, int64_t ncells,
                               const double* dts, double dt, double p, double* dstate, double* ddts, int J,
                               int64_t joff, int64_t jstride, double* jdst, int64_t jld, double* jdts, int* fb_list,
                               int* fb_count, unsigned long long* cnt) {
  cudaStream_t st = h->stream;
  const int nv = s->ns + 1;
  constexpr int kMax = tng_surrogate::kPipeChunks;
  int64_t chunk = (int64_t)1 << 18;
  if ((ncells + chunk - 1) / chunk > kMax) chunk = ((ncells + kMax - 1) / kMax + 127) / 128 * 128;
  const int nch = (int)((ncells + chunk - 1) / chunk);
  cudaError_t e = cudaSuccess;
  if (!s->copy_stream && (e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_error(e, "surrogate copy stream");
  for (auto& ev : s->pev)
    if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
      return cuda_error(e, "surrogate copy events");
  if (s->has_gate && !s->gout.reserve((size_t)ncells * s->gate.out_pad * sizeof(float)))
    return set_error(TNG_ERR_CUDA, "surrogate gate output allocation failed");
  // the uploads start after the handle's stream reached this point (the previous call may still
  // read the device buffers)
  cudaEventRecord(s->pev[0], st);
  cudaStreamWaitEvent(s->copy_stream, s->pev[0], 0);
  for (int k = 0; k < nch; ++k) {
    const int64_t a = k * chunk, n = std::min(chunk, ncells - a);
    cudaMemcpy2DAsync(dstate + a, ncells * sizeof(double), state + a, ld * sizeof(double), n * sizeof(double), nv,
                      cudaMemcpyHostToDevice, s->copy_stream);
    if (dts) cudaMemcpyAsync(ddts + a, dts + a, n * sizeof(double), cudaMemcpyHostToDevice, s->copy_stream);
    cudaEventRecord(s->pev[1 + k], s->copy_stream);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "surrogate state upload");
  cudaEventRecord(s->ev[0], st);
  for (int k = 0; k < nch; ++k) {
    const int64_t a = k * chunk, n = std::min(chunk, ncells - a);
    cudaStreamWaitEvent(st, s->pev[1 + k], 0);
    if (J > 0) {  // the judged cells of this chunk, before the post-processing overwrites them
      const int64_t j0 = a <= joff ? 0 : std::min<int64_t>(J, (a - joff + jstride - 1) / jstride);
      const int64_t j1 = std::min<int64_t>(J, (a + n - joff + jstride - 1) / jstride);
      if (j1 > j0)
        k_gather_cells<<<(int)((j1 - j0 + 127) / 128), 128, 0, st>>>(
            dstate, ncells, nv, (const int*)s->judge_idx.ptr + j0, (int)(j1 - j0), jdst + j0, jld, ddts, dt,
            jdts + j0);
    }
    float* out_k = (float*)s->out.ptr + (size_t)a * s->m.out_pad * s->members;
    int rc = launch_infer(h, s, dstate + a, n, ncells, ddts ? ddts + a : nullptr, dt, p, 0, s->members, out_k, true,
                          (int*)(cnt + 8), a);
    if (rc) return rc;
    SurPost pa = post_args(h, s, dstate + a, ncells, n, ddts ? ddts + a : nullptr, dt, p);
    pa.out = out_k;
    if (s->has_gate) pa.gate_out = (const float*)s->gout.ptr + a * s->gate.out_pad;
    pa.cell_base = (int)a;
    pa.fb_list = fb_list;
    pa.fb_count = fb_count;
    pa.cnt = cnt;
    k_sur_post<<<(int)std::min<int64_t>(4096, (n + 127) / 128), 128, 0, st>>>(pa);
  }
  cudaEventRecord(s->ev[1], st);
  cudaEventRecord(s->ev[2], st);
  e = cudaGetLastError();
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "surrogate kernels");
}

// The solved fallback cells into the host state: row v of the compact block (n cells, in list
// order) to state[v * ld + list[i]]. The cells are visited in increasing order (the list comes
// from atomics) and the species rows are split over a few threads.
static void scatter_fallback_host(double* state, int64_t ld, int nv, const double* comp, const int* list, int n) {
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return list[a] < list[b]; });
  const int nt = std::max(1, std::min<int>({nv, 8, (int)std::thread::hardware_concurrency()}));
  auto work = [&](int t) {
    for (int v = t; v < nv; v += nt) {
      double* row = state + (int64_t)v * ld;
      const double* src = comp + (int64_t)v * n;
      for (int i : ord) row[list[i]] = src[i];
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
}
}  // namespace tng

extern "C" {

void tng_surrogate_default_cfg(tng_surrogate_cfg* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->hidden = 256;
  c->layers = 4;
  c->seed = 20261203;
  c->ood_margin = 0.02;
  c->consist_tol_K = 5.0;
  c->clip_tol = 1e-3;
  c->judge_cells = 1024;
  c->post_mode = 1;
  c->target_mode = 1;
  c->members = 2;
  c->ens_tol_K = 2.f;
  c->ens_tol_Y = 5e-4f;
}

int tng_surrogate_create(tng_chem* h, const tng_surrogate_cfg* cfg, tng_surrogate** out) {
  if (!h || !out) return set_error(TNG_ERR_ARG, "tng_surrogate_create: null argument");
  *out = nullptr;
  tng_surrogate_cfg c;
  if (cfg)
    c = *cfg;
  else
    tng_surrogate_default_cfg(&c);
  if (c.members == 0) c.members = 2;
  if (!(c.ens_tol_K > 0.f)) c.ens_tol_K = 2.f;
  if (!(c.ens_tol_Y > 0.f)) c.ens_tol_Y = 5e-4f;
  if (c.members < 1 || c.members > kMaxMembers)
    return set_error(TNG_ERR_ARG, "tng_surrogate_create: 1..%d ensemble members", kMaxMembers);
  if (c.hidden != 256 || c.layers < 1 || c.layers > kMaxLayers - 1)
    return set_error(TNG_ERR_ARG, "tng_surrogate_create: hidden width must be 256 (the tensor-core tile), 1..%d layers",
                     kMaxLayers - 1);
  const MechOps* o = h->ops;
  if (o->ns > kPostNs || 2 * o->ns + 1 > 2 * kMaxNs || o->nelem + 1 > kMaxEl)
    return set_error(TNG_ERR_ARG, "tng_surrogate_create: mechanism too large (at most %d species, %d elements)",
                     kPostNs, kMaxEl);
  DeviceGuard g(h->cfg.device);
  tng_surrogate* s = new tng_surrogate();
  s->h = h;
  s->cfg = c;
  s->ns = o->ns;
  s->bath = 0;
  for (int k = 0; k < o->ns; ++k)
    if (std::strcmp(o->species[k], "N2") == 0) s->bath = k;
  s->n_in = 2 * o->ns + 1;  // T, log P, ns-1 species (log), log dt, ns-1 species (linear)
  s->n_out = o->ns + 1;
  s->nel = o->nelem;
  s->members = c.members;
  int rc = TNG_OK;
  for (int i = 0; i < s->members && !rc; ++i)
    rc = mlp_init(&s->member(i), h->cfg.device, h->stream, s->n_in, s->n_out, c.hidden, c.layers,
                  c.seed + 7919ULL * i);
  if (rc) {
    for (int i = 0; i < s->members; ++i) mlp_free(&s->member(i));
    delete s;
    return rc;
  }
  if (s->m.in_pad > 256 || s->m.out_pad > 256 || s->m.in_pad % 16 || s->m.out_pad % 16) {
    for (int i = 0; i < s->members; ++i) mlp_free(&s->member(i));
    delete s;
    return set_error(TNG_ERR_ARG, "tng_surrogate_create: unsupported layer widths");
  }
  cudaMalloc(&s->d_fnorm, sizeof(float) * 4 * s->m.in_pad);
  cudaMalloc(&s->d_tnorm, sizeof(double) * 2 * s->m.out_pad);
  for (int i = 0; i < s->members; ++i) cudaMalloc(&s->d_wpack[i], sizeof(__nv_bfloat16) * s->m.nparam);
  // element matrix per kg: a_ek / W_k (reference literal kinds of W_k)
  std::vector<double> E(s->nel * s->ns);
  const double* wm = o->wmol[h->cfg.literal_mode];
  for (int e = 0; e < s->nel; ++e)
    for (int k = 0; k < s->ns; ++k) E[e * s->ns + k] = o->elem[e * s->ns + k] / wm[k];
  cudaMalloc(&s->d_E, sizeof(double) * E.size());
  cudaMemcpy(s->d_E, E.data(), sizeof(double) * E.size(), cudaMemcpyHostToDevice);
  for (auto& ev : s->ev) cudaEventCreate(&ev);
  h->dependents++;
  s->fmean.assign(s->n_in, 0.0), s->fstd.assign(s->n_in, 1.0), s->fmin.assign(s->n_in, 0.0),
      s->fmax.assign(s->n_in, 0.0);
  s->tmean.assign(s->n_out, 0.0), s->tstd.assign(s->n_out, 1.0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    tng_surrogate_destroy(s);
    return cuda_error(e, "tng_surrogate_create");
  }
  *out = s;
  return TNG_OK;
}

int tng_surrogate_destroy(tng_surrogate* s) {
  if (!s) return TNG_OK;
  DeviceGuard g(s->m.device);
  cudaStreamSynchronize(s->m.stream);
  for (int i = 0; i < s->members; ++i) mlp_free(&s->member(i));
  if (s->has_gate) mlp_free(&s->gate);
  if (s->d_gpack) cudaFree(s->d_gpack);
  s->gout.release();
  if (s->d_fnorm) cudaFree(s->d_fnorm);
  if (s->d_tnorm) cudaFree(s->d_tnorm);
  if (s->d_E) cudaFree(s->d_E);
  for (auto* w : s->d_wpack)
    if (w) cudaFree(w);
  for (DevBuf* b : {&s->out, &s->fb, &s->cnt, &s->judge_state, &s->judge_dts, &s->judge_idx, &s->work, &s->joint})
    b->release();
  for (auto& ev : s->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : s->pev)
    if (ev) cudaEventDestroy(ev);
  for (auto ev : {s->ev_front, s->ev_down})
    if (ev) cudaEventDestroy(ev);
  if (s->h_comp) cudaFreeHost(s->h_comp);
  if (s->h_list) cudaFreeHost(s->h_list);
  if (s->copy_stream) {
    cudaStreamSynchronize(s->copy_stream);
    cudaStreamDestroy(s->copy_stream);
  }
  if (s->h) s->h->dependents--;
  delete s;
  return TNG_OK;
}

}  // extern "C"

namespace {

// Features and normalised targets of n pairs into s->work: X (n x in_pad), T (n x out_pad). With
// set_norm the normalisation (feature mean/std/range, target mean/std) is computed from these
// pairs and uploaded; otherwise the surrogate's stored normalisation is applied.
int sur_prepare_pairs(tng_surrogate* s, const double* state0, const double* state1, const double* dts, int64_t n,
                      int64_t ld, double p, bool set_norm, float** Xo, float** To) {
  const int ip = s->m.in_pad, op = s->m.out_pad;
  cudaStream_t st = s->m.stream;
  if (!s->work.reserve((size_t)n * (ip + op) * sizeof(float) + sizeof(double) * 4 * (ip + op) + 256 * sizeof(float)))
    return set_error(TNG_ERR_CUDA, "surrogate training: %lld pairs do not fit", (long long)n);
  float* X = (float*)s->work.ptr;
  float* T = X + (size_t)n * ip;
  double* stats = (double*)(T + (size_t)n * op);
  float* nrm = (float*)(stats + 4 * (ip + op));
  k_sur_features<<<1184, 128, 0, st>>>(state0, ld, (int)n, dts, std::log(p), s->ns, s->bath, ip, X);
  k_sur_targets<<<1184, 128, 0, st>>>(state0, state1, ld, (int)n, s->ns, op, T);
  if (set_norm) {
    k_colstats<<<ip, 256, 0, st>>>(X, (int)n, ip, stats);
    k_colstats<<<op, 256, 0, st>>>(T, (int)n, op, stats + 4 * ip);
    std::vector<double> hs(4 * (ip + op));
    cudaMemcpyAsync(hs.data(), stats, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "surrogate statistics");
    for (int i = 0; i < s->n_in; ++i) {
      const double mu = hs[4 * i] / n, var = std::max(hs[4 * i + 1] / n - mu * mu, 0.0);
      s->fmean[i] = mu;
      s->fstd[i] = std::max(std::sqrt(var), 1e-3 * std::max(1.0, std::fabs(mu)));
      s->fmin[i] = hs[4 * i + 2];
      s->fmax[i] = hs[4 * i + 3];
    }
    double shared = 0.0;  // target_mode 1: the RMS spread over the species outputs, one scale for all
    for (int i = 0; i < s->n_out; ++i) {
      const double* q = &hs[4 * (ip + i)];
      const double mu = q[0] / n, var = std::max(q[1] / n - mu * mu, 0.0);
      s->tmean[i] = mu;
      s->tstd[i] = std::max(std::sqrt(var), 1e-14);
      if (i > 0) shared += var;
    }
    if (s->cfg.target_mode == 1) {
      shared = std::max(std::sqrt(shared / std::max(1, s->n_out - 1)), 1e-14);
      for (int i = 1; i < s->n_out; ++i) s->tstd[i] = shared;
    }
    const int rc = sur_upload_norm(s);
    if (rc) return rc;
  }
  std::vector<float> hn(2 * (ip + op), 0.f);
  for (int i = 0; i < s->n_in; ++i) hn[i] = (float)s->fmean[i], hn[ip + i] = (float)(1.0 / s->fstd[i]);
  for (int i = 0; i < s->n_out; ++i)
    hn[2 * ip + i] = (float)s->tmean[i], hn[2 * ip + op + i] = (float)(1.0 / s->tstd[i]);
  cudaMemcpyAsync(nrm, hn.data(), sizeof(float) * hn.size(), cudaMemcpyHostToDevice, st);
  k_normalise<<<2048, 256, 0, st>>>(X, (int)n, ip, s->n_in, nrm, nrm + ip);
  k_normalise<<<2048, 256, 0, st>>>(T, (int)n, op, s->n_out, nrm + 2 * ip, nrm + 2 * ip + op);
  // the staged normalisation is read by the kernels above before the host vector goes away
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_error(e, "surrogate pairs");
  *Xo = X;
  *To = T;
  return TNG_OK;
}

// Errors of the current ensemble's post-processed prediction on n pairs, relative to the bars
// (k_sur_errors), into r (device, 2 floats per pair); predictions run in chunks.
int sur_pair_errors(tng_surrogate* s, const double* state0, const double* state1, const double* dts, int64_t n,
                    int64_t ld, double p, float* r) {
  const int nv = s->ns + 1;
  const int64_t chunk = std::min<int64_t>(n, 1 << 20);
  DevBuf tmp;
  if (!tmp.reserve((size_t)chunk * nv * sizeof(double))) return set_error(TNG_ERR_CUDA, "surrogate errors: scratch");
  int rc = TNG_OK;
  for (int64_t c0 = 0; c0 < n && !rc; c0 += chunk) {
    const int64_t m = std::min(chunk, n - c0);
    rc = tng_surrogate_predict(s->h, s, state0 + c0, m, ld, dts + c0, 0.0, p, (double*)tmp.ptr, m, nullptr, nullptr);
    if (rc) break;
    k_sur_errors<<<(int)std::min<int64_t>(4096, (m + 127) / 128), 128, 0, s->h->stream>>>(
        (const double*)tmp.ptr, m, state1 + c0, ld, (int)m, s->ns, r + 2 * c0);
    cudaError_t e = cudaStreamSynchronize(s->h->stream);
    if (e != cudaSuccess) rc = cuda_error(e, "surrogate errors");
  }
  tmp.release();
  return rc;
}

}  // namespace

extern "C" {

int tng_surrogate_train(tng_surrogate* s, const double* state0, const double* state1, const double* dts, int64_t n,
                        int64_t ld, double p, int epochs, int batch, double lr, float* losses) {
  if (!s || !state0 || !state1 || !dts || n < 16 || ld < n || !(p > 0.0) || n > (1LL << 31) - 1)
    return set_error(TNG_ERR_ARG, "tng_surrogate_train: bad argument");
  DeviceGuard g(s->m.device);
  const int op = s->m.out_pad;
  cudaStream_t st = s->m.stream;
  float *X, *T;
  int rc = sur_prepare_pairs(s, state0, state1, dts, n, ld, p, true, &X, &T);
  if (rc) return rc;
  // loss weights: every species output equally (outputs are normalised), temperature wT
  std::vector<float> w(op, 0.f);
  const float wT = s->cfg.loss_T_weight > 0.f ? s->cfg.loss_T_weight : 2.f;
  for (int i = 0; i < s->n_out; ++i) w[i] = i == 0 ? wT : 1.f;
  float* dw;
  cudaError_t e;
  if ((e = cudaMalloc(&dw, sizeof(float) * op)) != cudaSuccess) return cuda_error(e, "loss weights");
  cudaMemcpyAsync(dw, w.data(), sizeof(float) * op, cudaMemcpyHostToDevice, st);
  // every member on the same normalised pairs, from its own initialisation and shuffling order;
  // the reported loss is the members' mean per epoch
  std::vector<float> lm(epochs > 0 ? epochs : 1);
  if (losses) std::fill(losses, losses + epochs, 0.f);
  for (int i = 0; i < s->members && !rc; ++i) {
    rc = mlp_train(&s->member(i), X, T, dw, n, epochs, batch, (float)lr, s->cfg.seed + 1 + 104729ULL * i, lm.data());
    if (losses)
      for (int ep = 0; ep < epochs; ++ep) losses[ep] += lm[ep] / s->members;
  }
  cudaStreamSynchronize(st);
  cudaFree(dw);
  if (rc) return rc;
  if ((rc = sur_pack(s))) return rc;
  s->trained = true;
  return TNG_OK;
}

int tng_surrogate_refine(tng_surrogate* s, const double* state0, const double* state1, const double* dts, int64_t n,
                         int64_t ld, double p, int epochs, int batch, double lr, double boost, float* losses,
                         int64_t* population) {
  if (!s || !state0 || !state1 || !dts || n < 16 || ld < n || !(p > 0.0) || n > (1LL << 31) - 1 || epochs < 1 ||
      !(boost >= 0.0))
    return set_error(TNG_ERR_ARG, "tng_surrogate_refine: bad argument");
  if (!s->trained) return set_error(TNG_ERR_STATE, "tng_surrogate_refine: surrogate not trained or loaded");
  DeviceGuard g(s->m.device);
  cudaStream_t st = s->m.stream;
  float* r;
  cudaError_t e = cudaMalloc(&r, sizeof(float) * 2 * n);
  if (e != cudaSuccess) return cuda_error(e, "tng_surrogate_refine: errors");
  int rc = sur_pair_errors(s, state0, state1, dts, n, ld, p, r);
  std::vector<float> hr(2 * (size_t)n);
  if (!rc) {
    e = cudaMemcpy(hr.data(), r, sizeof(float) * hr.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_error(e, "tng_surrogate_refine: errors");
  }
  cudaFree(r);
  if (rc) return rc;
  // the resampled population: pair i appears 1 + min(round(boost * e_i), 16) times, e_i its
  // larger error relative to the bars
  std::vector<int> pop;
  pop.reserve((size_t)n + n / 4);
  for (int64_t i = 0; i < n; ++i) {
    const float ei = std::max(hr[2 * i], hr[2 * i + 1]);
    const int reps = 1 + (std::isfinite(ei) ? (int)std::min(16.0, std::nearbyint(boost * ei)) : 16);
    for (int k = 0; k < reps; ++k) pop.push_back((int)i);
  }
  if (population) *population = (int64_t)pop.size();
  float *X, *T;
  if ((rc = sur_prepare_pairs(s, state0, state1, dts, n, ld, p, false, &X, &T))) return rc;
  const int op = s->m.out_pad;
  std::vector<float> w(op, 0.f);
  const float wT = s->cfg.loss_T_weight > 0.f ? s->cfg.loss_T_weight : 2.f;
  for (int i = 0; i < s->n_out; ++i) w[i] = i == 0 ? wT : 1.f;
  float* dw;
  if ((e = cudaMalloc(&dw, sizeof(float) * op)) != cudaSuccess) return cuda_error(e, "loss weights");
  cudaMemcpyAsync(dw, w.data(), sizeof(float) * op, cudaMemcpyHostToDevice, st);
  std::vector<float> lm(epochs);
  if (losses) std::fill(losses, losses + epochs, 0.f);
  for (int i = 0; i < s->members && !rc; ++i) {
    rc = mlp_train(&s->member(i), X, T, dw, n, epochs, batch, (float)lr, s->cfg.seed + 77 + 104729ULL * i, lm.data(),
                   pop.data(), (int64_t)pop.size());
    if (losses)
      for (int ep = 0; ep < epochs; ++ep) losses[ep] += lm[ep] / s->members;
  }
  cudaStreamSynchronize(st);
  cudaFree(dw);
  if (rc) return rc;
  return sur_pack(s);
}

int tng_surrogate_train_gate(tng_surrogate* s, const double* state0, const double* state1, const double* dts,
                             int64_t n, int64_t ld, double p, int epochs, int batch, double lr, double under,
                             float* losses) {
  if (!s || !state0 || !state1 || !dts || n < 16 || ld < n || !(p > 0.0) || n > (1LL << 31) - 1 || epochs < 1 ||
      !(under > 0.0))
    return set_error(TNG_ERR_ARG, "tng_surrogate_train_gate: bad argument");
  if (!s->trained) return set_error(TNG_ERR_STATE, "tng_surrogate_train_gate: surrogate not trained or loaded");
  DeviceGuard g(s->m.device);
  cudaStream_t st = s->m.stream;
  int rc;
  if (!s->has_gate) {
    if ((rc = mlp_init(&s->gate, s->m.device, st, s->n_in, 2, s->cfg.hidden, s->cfg.layers, s->cfg.seed + 424242ULL)))
      return rc;
    cudaError_t e = cudaMalloc(&s->d_gpack, sizeof(__nv_bfloat16) * s->gate.nparam);
    if (e != cudaSuccess) {
      mlp_free(&s->gate);
      return cuda_error(e, "tng_surrogate_train_gate: packed weights");
    }
    s->has_gate = true;
  }
  const int gp = s->gate.out_pad;
  // errors of the members (the gate's own verdict plays no part in them)
  float* r;
  float* Tg;
  cudaError_t e = cudaMalloc(&r, sizeof(float) * 2 * n);
  if (e != cudaSuccess) return cuda_error(e, "tng_surrogate_train_gate: errors");
  if ((e = cudaMalloc(&Tg, sizeof(float) * (size_t)n * gp + sizeof(double) * 4 * gp + 64)) != cudaSuccess) {
    cudaFree(r);
    return cuda_error(e, "tng_surrogate_train_gate: targets");
  }
  rc = sur_pair_errors(s, state0, state1, dts, n, ld, p, r);
  float *X = nullptr, *T = nullptr;
  if (!rc) rc = sur_prepare_pairs(s, state0, state1, dts, n, ld, p, false, &X, &T);
  if (!rc) {
    double* gst = (double*)(Tg + (size_t)n * gp);
    k_gate_targets<<<1184, 128, 0, st>>>(r, (int)n, gp, Tg);
    k_colstats<<<2, 256, 0, st>>>(Tg, (int)n, gp, gst);
    double hs[8];
    cudaMemcpyAsync(hs, gst, sizeof(hs), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) rc = cuda_error(e, "gate statistics");
    if (!rc) {
      std::vector<float> hn(2 * gp, 0.f);
      for (int i = 0; i < 2; ++i) {
        const double mu = hs[4 * i] / n, var = std::max(hs[4 * i + 1] / n - mu * mu, 0.0);
        s->gate_mean[i] = mu;
        s->gate_std[i] = std::max(std::sqrt(var), 1e-3);
        hn[i] = (float)mu;
        hn[gp + i] = (float)(1.0 / s->gate_std[i]);
      }
      float* dn = (float*)(gst + 2 * 4);
      cudaMemcpyAsync(dn, hn.data(), sizeof(float) * hn.size(), cudaMemcpyHostToDevice, st);
      k_normalise<<<2048, 256, 0, st>>>(Tg, (int)n, gp, 2, dn, dn + gp);
      std::vector<float> w(gp, 0.f);
      w[0] = w[1] = 1.f;
      float* dw = dn + 2 * gp;
      cudaMemcpyAsync(dw, w.data(), sizeof(float) * gp, cudaMemcpyHostToDevice, st);
      s->gate.under_weight = (float)under;
      rc = mlp_train(&s->gate, X, Tg, dw, n, epochs, batch, (float)lr, s->cfg.seed + 99991ULL, losses);
      cudaStreamSynchronize(st);
    }
  }
  cudaFree(r);
  cudaFree(Tg);
  if (rc) return rc;
  return sur_pack(s);
}

int tng_surrogate_set_gate_tol(tng_surrogate* s, double tol) {
  if (!s || !(tol > 0.0)) return set_error(TNG_ERR_ARG, "tng_surrogate_set_gate_tol: bad argument");
  if (!s->has_gate) return set_error(TNG_ERR_STATE, "tng_surrogate_set_gate_tol: the surrogate has no error gate");
  s->gate_tol = tol;
  return TNG_OK;
}

int tng_surrogate_gate_info(const tng_surrogate* s, int* has_gate, double* tol) {
  if (!s) return set_error(TNG_ERR_ARG, "tng_surrogate_gate_info: null handle");
  if (has_gate) *has_gate = s->has_gate ? 1 : 0;
  if (tol) *tol = s->cfg.gate_tol > 0.f ? (double)s->cfg.gate_tol : s->gate_tol;
  return TNG_OK;
}

int tng_surrogate_save(const tng_surrogate* s, const char* path) {
  if (!s || !path) return set_error(TNG_ERR_ARG, "tng_surrogate_save: null argument");
  if (!s->trained) return set_error(TNG_ERR_STATE, "tng_surrogate_save: surrogate not trained");
  std::vector<float> params(s->m.nparam * s->members);
  std::vector<float> gparams(s->has_gate ? s->gate.nparam : 0);
  DeviceGuard g(s->m.device);
  cudaStreamSynchronize(s->m.stream);
  for (int i = 0; i < s->members; ++i)
    cudaMemcpy(params.data() + i * s->m.nparam, s->member(i).params, sizeof(float) * s->m.nparam,
               cudaMemcpyDeviceToHost);
  if (s->has_gate) cudaMemcpy(gparams.data(), s->gate.params, sizeof(float) * s->gate.nparam, cudaMemcpyDeviceToHost);
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(TNG_ERR_ARG, "tng_surrogate_save: cannot open %s", path);
  char magic[8] = {'T', 'N', 'G', 'S', 'U', 'R', '3', 0};
  char mech[32] = {};
  std::snprintf(mech, sizeof(mech), "%s", s->h->ops->name);
  int hdr[10] = {s->ns, s->n_in, s->n_out, s->cfg.hidden, s->cfg.layers, s->bath, s->h->cfg.literal_mode, s->members,
                 s->has_gate ? 1 : 0, 0};
  int64_t np = s->m.nparam;
  bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(mech, 1, 32, f) == 32 && std::fwrite(hdr, 4, 10, f) == 10 &&
            std::fwrite(&np, 8, 1, f) == 1;
  for (const std::vector<double>* v : {&s->fmean, &s->fstd, &s->fmin, &s->fmax, &s->tmean, &s->tstd})
    ok = ok && std::fwrite(v->data(), 8, v->size(), f) == v->size();
  ok = ok && std::fwrite(params.data(), 4, params.size(), f) == params.size();
  if (s->has_gate) {
    const int64_t gnp = s->gate.nparam;
    const double gd[5] = {s->gate_mean[0], s->gate_mean[1], s->gate_std[0], s->gate_std[1], s->gate_tol};
    ok = ok && std::fwrite(&gnp, 8, 1, f) == 1 && std::fwrite(gd, 8, 5, f) == 5 &&
         std::fwrite(gparams.data(), 4, gparams.size(), f) == gparams.size();
  }
  std::fclose(f);
  return ok ? TNG_OK : set_error(TNG_ERR_ARG, "tng_surrogate_save: write failed");
}

int tng_surrogate_load(tng_surrogate* s, const char* path) {
  if (!s || !path) return set_error(TNG_ERR_ARG, "tng_surrogate_load: null argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(TNG_ERR_ARG, "tng_surrogate_load: cannot open %s", path);
  char magic[8], mech[32];
  int hdr[10] = {};
  int64_t np = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::fread(mech, 1, 32, f) == 32;
  // TNGSUR2: 8 header ints, no gate; TNGSUR3: 10 header ints, hdr[8] = gate present
  const bool v3 = ok && std::memcmp(magic, "TNGSUR3", 8) == 0;
  if (!ok || (!v3 && std::memcmp(magic, "TNGSUR2", 8) != 0)) {
    std::fclose(f);
    return set_error(TNG_ERR_ARG, "tng_surrogate_load: %s is not a surrogate file", path);
  }
  const int nh = v3 ? 10 : 8;
  ok = std::fread(hdr, 4, nh, f) == (size_t)nh && std::fread(&np, 8, 1, f) == 1;
  mech[31] = 0;
  if (!ok || std::strcmp(mech, s->h->ops->name) != 0 || hdr[0] != s->ns || hdr[1] != s->n_in || hdr[2] != s->n_out ||
      hdr[3] != s->cfg.hidden || hdr[4] != s->cfg.layers || np != s->m.nparam) {
    std::fclose(f);
    return set_error(TNG_ERR_ARG, "tng_surrogate_load: %s was trained for %s with other sizes", path, mech);
  }
  if (hdr[7] != s->members) {
    std::fclose(f);
    return set_error(TNG_ERR_ARG, "tng_surrogate_load: %s holds %d ensemble members, the surrogate was created with %d",
                     path, hdr[7], s->members);
  }
  for (std::vector<double>* v : {&s->fmean, &s->fstd, &s->fmin, &s->fmax, &s->tmean, &s->tstd})
    ok = ok && std::fread(v->data(), 8, v->size(), f) == v->size();
  std::vector<float> params(np * s->members);
  ok = ok && std::fread(params.data(), 4, params.size(), f) == params.size();
  const bool gate = v3 && hdr[8] == 1;
  std::vector<float> gparams;
  double gd[5] = {0.0, 0.0, 1.0, 1.0, 0.25};
  int64_t gnp = 0;
  if (ok && gate) {
    ok = std::fread(&gnp, 8, 1, f) == 1 && std::fread(gd, 8, 5, f) == 5 && gnp > 0 && gnp < (1LL << 30);
    if (ok) {
      gparams.resize(gnp);
      ok = std::fread(gparams.data(), 4, gparams.size(), f) == gparams.size();
    }
  }
  std::fclose(f);
  if (!ok) return set_error(TNG_ERR_ARG, "tng_surrogate_load: %s is truncated", path);
  DeviceGuard g(s->m.device);
  for (int i = 0; i < s->members; ++i)
    cudaMemcpy(s->member(i).params, params.data() + i * np, sizeof(float) * np, cudaMemcpyHostToDevice);
  if (gate) {
    if (!s->has_gate) {
      int rc = mlp_init(&s->gate, s->m.device, s->m.stream, s->n_in, 2, s->cfg.hidden, s->cfg.layers, 0);
      if (rc) return rc;
      cudaError_t e = cudaMalloc(&s->d_gpack, sizeof(__nv_bfloat16) * s->gate.nparam);
      if (e != cudaSuccess) {
        mlp_free(&s->gate);
        return cuda_error(e, "tng_surrogate_load: gate weights");
      }
      s->has_gate = true;
    }
    if (gnp != s->gate.nparam) return set_error(TNG_ERR_ARG, "tng_surrogate_load: %s: gate of another size", path);
    cudaMemcpy(s->gate.params, gparams.data(), sizeof(float) * gnp, cudaMemcpyHostToDevice);
    s->gate_mean[0] = gd[0], s->gate_mean[1] = gd[1], s->gate_std[0] = gd[2], s->gate_std[1] = gd[3];
    s->gate_tol = gd[4];
  }
  int rc = sur_upload_norm(s);
  if (rc) return rc;
  if ((rc = sur_pack(s))) return rc;
  cudaError_t e = cudaStreamSynchronize(s->m.stream);
  if (e != cudaSuccess) return cuda_error(e, "tng_surrogate_load");
  s->trained = true;
  return TNG_OK;
}

int tng_surrogate_debug_waits(tng_surrogate* s, int wait_limit, int fault) {
  if (!s || wait_limit < 0 || fault < 0 || fault > 1)
    return set_error(TNG_ERR_ARG, "tng_surrogate_debug_waits: bad argument");
  s->dbg_wait_limit = wait_limit;
  s->dbg_fault = fault;
  return TNG_OK;
}

int tng_surrogate_dims(const tng_surrogate* s, int* n_in, int* n_out, int* in_pad, int* out_pad, int64_t* nparam) {
  if (!s) return set_error(TNG_ERR_ARG, "tng_surrogate_dims: null handle");
  if (n_in) *n_in = s->n_in;
  if (n_out) *n_out = s->n_out;
  if (in_pad) *in_pad = s->m.in_pad;
  if (out_pad) *out_pad = s->m.out_pad;
  if (nparam) *nparam = s->m.nparam;
  return TNG_OK;
}

int tng_surrogate_params(tng_surrogate* s, float* host, int set) {
  if (!s || !host) return set_error(TNG_ERR_ARG, "tng_surrogate_params: null argument");
  DeviceGuard g(s->m.device);
  cudaStreamSynchronize(s->m.stream);
  cudaError_t e;
  if (set) {
    e = cudaMemcpy(s->m.params, host, sizeof(float) * s->m.nparam, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && s->trained) {
      int rc = sur_pack(s);
      if (rc) return rc;
      e = cudaStreamSynchronize(s->m.stream);
    }
  } else {
    e = cudaMemcpy(host, s->m.params, sizeof(float) * s->m.nparam, cudaMemcpyDeviceToHost);
  }
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "tng_surrogate_params");
}

int tng_surrogate_features(tng_surrogate* s, const double* state, int64_t n, int64_t ld, const double* dts, double p,
                           float* X) {
  if (!s || !state || !dts || !X || n <= 0 || ld < n) return set_error(TNG_ERR_ARG, "tng_surrogate_features: bad argument");
  DeviceGuard g(s->m.device);
  const int ip = s->m.in_pad;
  k_sur_features<<<1184, 128, 0, s->m.stream>>>(state, ld, (int)n, dts, std::log(p), s->ns, s->bath, ip, X);
  std::vector<float> hn(2 * ip, 0.f);
  for (int i = 0; i < s->n_in; ++i) hn[i] = (float)s->fmean[i], hn[ip + i] = (float)(1.0 / s->fstd[i]);
  float* dn;
  cudaError_t e = cudaMalloc(&dn, sizeof(float) * 2 * ip);
  if (e != cudaSuccess) return cuda_error(e, "tng_surrogate_features");
  cudaMemcpyAsync(dn, hn.data(), sizeof(float) * 2 * ip, cudaMemcpyHostToDevice, s->m.stream);
  k_normalise<<<1024, 256, 0, s->m.stream>>>(X, (int)n, ip, s->n_in, dn, dn + ip);
  e = cudaStreamSynchronize(s->m.stream);
  cudaFree(dn);
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "tng_surrogate_features");
}

int tng_surrogate_forward_f32(tng_surrogate* s, const float* X, int64_t n, float* Y) {
  if (!s || !X || !Y || n <= 0 || n > (1 << 24)) return set_error(TNG_ERR_ARG, "tng_surrogate_forward_f32: bad argument");
  DeviceGuard g(s->m.device);
  float* out;
  int rc = mlp_forward_f32(&s->m, X, (int)n, &out);
  if (rc) return rc;
  cudaMemcpyAsync(Y, out, sizeof(float) * n * s->m.out_pad, cudaMemcpyDeviceToDevice, s->m.stream);
  cudaError_t e = cudaStreamSynchronize(s->m.stream);
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "tng_surrogate_forward_f32");
}

int tng_surrogate_infer(tng_surrogate* s, const double* state, int64_t n, int64_t ld, const double* dts, double dt,
                        double p, float* out) {
  if (!s || !state || !out || n <= 0 || ld < n) return set_error(TNG_ERR_ARG, "tng_surrogate_infer: bad argument");
  if (!s->trained) return set_error(TNG_ERR_STATE, "tng_surrogate_infer: surrogate not trained or loaded");
  DeviceGuard g(s->m.device);
  if (!s->cnt.reserve(16 * sizeof(unsigned long long))) return set_error(TNG_ERR_CUDA, "scratch");
  int* err = (int*)((unsigned long long*)s->cnt.ptr + 8);
  cudaMemsetAsync(err, 0, sizeof(int), s->m.stream);
  int rc = launch_infer(s->h, s, state, n, ld, dts, dt, p, 0, 1, out, false, err);
  if (rc) return rc;
  int herr = 0;
  cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s->m.stream);
  cudaError_t e = cudaStreamSynchronize(s->m.stream);
  if (e != cudaSuccess) return cuda_error(e, "tng_surrogate_infer");
  if (herr) return set_error(TNG_ERR_CUDA, "tng_surrogate_infer: tensor-core inference timed out");
  return TNG_OK;
}

int tng_substep_surrogate(tng_chem* h, tng_surrogate* s, double* state, int64_t ncells, int64_t ld, const double* dts,
                          double dt, double p, int flags, tng_surrogate_stats* stats) {
  if (!h || !s || s->h != h) return set_error(TNG_ERR_ARG, "tng_substep_surrogate: handle/surrogate mismatch");
  if (!s->trained) return set_error(TNG_ERR_STATE, "tng_substep_surrogate: surrogate not trained or loaded");
  if (ncells < 0 || ld < ncells || ncells > (1LL << 31) - 1)
    return set_error(TNG_ERR_ARG, "tng_substep_surrogate: need 0 <= ncells <= ld < 2^31");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (ncells == 0) return TNG_OK;
  if (!state || !(p > 0.0) || (!dts && !(dt >= 0.0))) return set_error(TNG_ERR_ARG, "tng_substep_surrogate: bad argument");
  if (flags != TNG_DEVICE_PTRS && flags != TNG_HOST_PTRS) return set_error(TNG_ERR_ARG, "tng_substep_surrogate: bad flags");
  DeviceGuard g(h->cfg.device);
  cudaStream_t st = h->stream;
  const int nv = s->ns + 1;
  cudaError_t e;
  // with host pointers and a large batch the upload is overlapped with the front of the substep
  const bool pipelined = flags == TNG_HOST_PTRS && ncells >= ((int64_t)1 << 19);
  double* dstate = state;
  const double* ddts = dts;
  int64_t dld = ld;
  if (flags == TNG_HOST_PTRS) {
    if (!h->bufs[6].reserve((size_t)nv * ncells * sizeof(double)) ||
        (dts && !h->bufs[7].reserve(ncells * sizeof(double))))
      return set_error(TNG_ERR_CUDA, "tng_substep_surrogate: device state allocation failed");
    dstate = (double*)h->bufs[6].ptr;
    dld = ncells;
    if (dts) ddts = (const double*)h->bufs[7].ptr;
    if (!pipelined) {
      cudaMemcpy2DAsync(dstate, ncells * sizeof(double), state, ld * sizeof(double), ncells * sizeof(double), nv,
                        cudaMemcpyHostToDevice, st);
      if (dts) cudaMemcpyAsync(h->bufs[7].ptr, dts, ncells * sizeof(double), cudaMemcpyHostToDevice, st);
    }
  }
  const int J = (int)std::min<int64_t>(ncells, std::max(0, s->cfg.judge_cells));
  bool ok = s->out.reserve((size_t)ncells * s->m.out_pad * s->members * sizeof(float)) && s->fb.reserve((ncells + 1) * sizeof(int)) &&
            s->cnt.reserve(16 * sizeof(unsigned long long)) &&
            (J == 0 || (s->judge_state.reserve((size_t)J * nv * sizeof(double)) &&
                        s->judge_dts.reserve((size_t)J * sizeof(double)) && s->judge_idx.reserve(J * sizeof(int))));
  // With statistics requested the judged sample and the fallback cells are solved in ONE launch of
  // the implicit solver (a joint batch: the sample in columns 0..J-1, the fallback cells after
  // it), so the two tails overlap instead of adding up.
  const bool joint = J > 0 && stats;
  const int64_t ldc = J + ncells;
  double* comp = nullptr;
  double* comp_dts = nullptr;
  int* comp_iota = nullptr;
  int* comp_n = nullptr;
  if (ok && joint) {
    ok = s->joint.reserve((size_t)ldc * (nv + 1) * sizeof(double) + (size_t)(ldc + 4) * sizeof(int));
    comp = (double*)s->joint.ptr;
    comp_dts = comp + (size_t)nv * ldc;
    comp_iota = (int*)(comp_dts + ldc);
    comp_n = comp_iota + ldc;
  }
  if (!ok) return set_error(TNG_ERR_CUDA, "tng_substep_surrogate: scratch allocation failed");
  int rc = solver_prepare(h);  // the solver tables (thermo for the enthalpy balance) on the device
  if (rc) return rc;
  int* fb_count = (int*)s->fb.ptr;
  int* fb_list = fb_count + 1;
  unsigned long long* cnt = (unsigned long long*)s->cnt.ptr;
  cudaMemsetAsync(fb_count, 0, sizeof(int), st);
  cudaMemsetAsync(cnt, 0, 16 * sizeof(unsigned long long), st);
  // held-out sample: a strided set of cells that rotates from call to call
  if (J > 0) {
    std::vector<int> idx(J);
    const int64_t stride = std::max<int64_t>(1, ncells / J);
    const int64_t off = (int64_t)(s->calls * 7919) % stride;
    for (int j = 0; j < J; ++j) idx[j] = (int)((off + (int64_t)j * stride) % ncells);
    cudaMemcpyAsync(s->judge_idx.ptr, idx.data(), sizeof(int) * J, cudaMemcpyHostToDevice, st);
    if (pipelined)
      ;  // gathered chunk by chunk below
    else if (joint)
      k_gather_cells<<<(J + 127) / 128, 128, 0, st>>>(dstate, dld, nv, (const int*)s->judge_idx.ptr, J, comp, ldc,
                                                      ddts, dt, comp_dts);
    else
      k_gather_cells<<<(J + 127) / 128, 128, 0, st>>>(dstate, dld, nv, (const int*)s->judge_idx.ptr, J,
                                                      (double*)s->judge_state.ptr, J, ddts, dt,
                                                      (double*)s->judge_dts.ptr);
  }
  s->calls++;
  if (pipelined) {
    const int64_t jstride = J > 0 ? std::max<int64_t>(1, ncells / J) : 1;
    const int64_t joff = J > 0 ? (int64_t)((s->calls - 1) * 7919) % jstride : 0;
    rc = sur_front_pipelined(h, s, state, ld, ncells, dts, dt, p, dstate, (double*)ddts, J, joff, jstride,
                             joint ? comp : (double*)s->judge_state.ptr, joint ? ldc : J,
                             joint ? comp_dts : (double*)s->judge_dts.ptr, fb_list, fb_count, cnt);
    if (rc) return rc;
    if (joint) {
      // every accepted cell is final now: the state goes back during the fallback solve, which
      // works on its own batch (the fallback cells are patched on the host afterwards)
      for (auto* ev : {&s->ev_front, &s->ev_down})
        if (!*ev && (e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess)
          return cuda_error(e, "surrogate download events");
      cudaEventRecord(s->ev_front, st);
      cudaStreamWaitEvent(s->copy_stream, s->ev_front, 0);
      cudaMemcpy2DAsync(state, ld * sizeof(double), dstate, ncells * sizeof(double), ncells * sizeof(double), nv,
                        cudaMemcpyDeviceToHost, s->copy_stream);
      cudaEventRecord(s->ev_down, s->copy_stream);
    }
  } else {
    // inference on the tensor cores
    cudaEventRecord(s->ev[0], st);
    rc = launch_infer(h, s, dstate, ncells, dld, ddts, dt, p, 0, s->members, (float*)s->out.ptr, true,
                      (int*)(cnt + 8));
    if (rc) return rc;
    cudaEventRecord(s->ev[1], st);
    // post-processing and fallback list
    SurPost pa = post_args(h, s, dstate, dld, ncells, ddts, dt, p);
    pa.fb_list = fb_list;
    pa.fb_count = fb_count;
    pa.cnt = cnt;
    k_sur_post<<<(int)std::min<int64_t>(4096, (ncells + 127) / 128), 128, 0, st>>>(pa);
    cudaEventRecord(s->ev[2], st);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "surrogate kernels");
  }
  tng_substep_stats fst;
  if (joint) {
    // fallback cells and the judged sample in one implicit solve, then the fallback cells back
    k_gather_list<<<1184, 128, 0, st>>>(dstate, dld, nv, fb_list, fb_count, J, comp, ldc, ddts, dt, comp_dts, comp_n);
    k_joint_order<<<(int)std::min<int64_t>(4096, (ldc + 255) / 256), 256, 0, st>>>(comp_iota, fb_count, J, ldc);
    rc = substep_run(h, comp, ldc, ldc, comp_dts, 0.0, p, TNG_DEVICE_PTRS, comp_iota, comp_n, nullptr, nullptr, nullptr,
                     &fst);
    if (rc) {
      if (pipelined) cudaStreamSynchronize(s->copy_stream);  // no copy into the caller's buffer after return
      return rc;
    }
    if (pipelined) cudaStreamWaitEvent(st, s->ev_down, 0);  // the download has read the state
    k_scatter_list<<<1184, 128, 0, st>>>(dstate, dld, nv, fb_list, fb_count, J, comp, ldc);
    cudaEventRecord(s->ev[3], st);
    // judge: the implicit solve of the sample against the surrogate(+fallback) result
    k_judge<<<(J + 127) / 128, 128, 0, st>>>(dstate, dld, s->ns, (const int*)s->judge_idx.ptr, J, comp, ldc,
                                             (double*)(cnt + 10));
  } else {
    // implicit fallback on the listed cells, in place
    rc = substep_run(h, dstate, ncells, dld, ddts, dt, p, TNG_DEVICE_PTRS, fb_list, fb_count, nullptr, nullptr,
                     nullptr, stats ? &fst : nullptr);
    if (rc) return rc;
    cudaEventRecord(s->ev[3], st);
  }
  cudaEventRecord(s->ev[4], st);
  const bool patch = pipelined && joint;  // download overlapped, fallback cells patched on the host
  if (flags == TNG_HOST_PTRS && !patch)
    cudaMemcpy2DAsync(state, ld * sizeof(double), dstate, ncells * sizeof(double), ncells * sizeof(double), nv,
                      cudaMemcpyDeviceToHost, st);
  if (stats || flags == TNG_HOST_PTRS) {
    unsigned long long hc[16];
    int nfb = 0;
    cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st);
    if (patch) cudaMemcpyAsync(&nfb, fb_count, sizeof(int), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (patch && (e != cudaSuccess || hc[8])) cudaStreamSynchronize(s->copy_stream);
    if (e != cudaSuccess) return cuda_error(e, "surrogate substep");
    if (hc[8]) return set_error(TNG_ERR_CUDA, "tng_substep_surrogate: tensor-core inference timed out");
    if (patch) {
      if (nfb > 0) {
        if ((size_t)nfb > s->h_cap) {
          if (s->h_comp) cudaFreeHost(s->h_comp);
          if (s->h_list) cudaFreeHost(s->h_list);
          s->h_comp = nullptr, s->h_list = nullptr, s->h_cap = 0;
          if ((e = cudaMallocHost(&s->h_comp, (size_t)nfb * nv * sizeof(double))) != cudaSuccess ||
              (e = cudaMallocHost(&s->h_list, (size_t)nfb * sizeof(int))) != cudaSuccess) {
            cudaStreamSynchronize(s->copy_stream);
            return cuda_error(e, "surrogate fallback staging");
          }
          s->h_cap = (size_t)nfb;
        }
        cudaMemcpy2DAsync(s->h_comp, (size_t)nfb * sizeof(double), comp + J, ldc * sizeof(double),
                          (size_t)nfb * sizeof(double), nv, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(s->h_list, fb_list, (size_t)nfb * sizeof(int), cudaMemcpyDeviceToHost, st);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
          cudaStreamSynchronize(s->copy_stream);
          return cuda_error(e, "surrogate fallback download");
        }
      }
      if ((e = cudaEventSynchronize(s->ev_down)) != cudaSuccess) return cuda_error(e, "surrogate state download");
      if (nfb > 0) scatter_fallback_host(state, ld, nv, s->h_comp, s->h_list, nfb);
    }
    if (stats) {
      stats->cells = ncells;
      stats->accepted = (int64_t)hc[0];
      stats->fallback_ood = (int64_t)hc[1];
      stats->fallback_consistency = (int64_t)hc[2];
      stats->fallback_clip = (int64_t)hc[3];
      stats->judged = J;
      double jd[2];
      std::memcpy(jd, &hc[10], sizeof(jd));
      stats->judge_max_rel_dT = jd[0];
      stats->judge_max_dY = jd[1];
      float a = 0, b = 0, c = 0, d = 0;
      cudaEventElapsedTime(&a, s->ev[0], s->ev[1]);
      cudaEventElapsedTime(&b, s->ev[1], s->ev[2]);
      cudaEventElapsedTime(&c, s->ev[2], s->ev[3]);
      cudaEventElapsedTime(&d, s->ev[0], s->ev[3]);
      stats->ms_infer = a, stats->ms_post = b, stats->ms_fallback = c, stats->ms_total = d;
      stats->fallback = fst;
      stats->fallback.cells = (int64_t)(hc[1] + hc[2] + hc[3] + hc[4] + hc[5]);
      stats->fallback_ensemble = (int64_t)hc[4];
      stats->fallback_gate = (int64_t)hc[5];
    }
  }
  return TNG_OK;
}

int tng_surrogate_predict(tng_chem* h, tng_surrogate* s, const double* state, int64_t ncells, int64_t ld,
                          const double* dts, double dt, double p, double* out, int64_t ld_out, int* reason,
                          double* indicator) {
  if (!h || !s || s->h != h) return set_error(TNG_ERR_ARG, "tng_surrogate_predict: handle/surrogate mismatch");
  if (!s->trained) return set_error(TNG_ERR_STATE, "tng_surrogate_predict: surrogate not trained or loaded");
  if (ncells < 0 || ld < ncells || ld_out < ncells || ncells > (1LL << 31) - 1)
    return set_error(TNG_ERR_ARG, "tng_surrogate_predict: need 0 <= ncells <= ld, ld_out < 2^31");
  if (ncells == 0) return TNG_OK;
  if (!state || !out || !(p > 0.0) || (!dts && !(dt >= 0.0)))
    return set_error(TNG_ERR_ARG, "tng_surrogate_predict: bad argument");
  DeviceGuard g(h->cfg.device);
  cudaStream_t st = h->stream;
  if (!s->out.reserve((size_t)ncells * s->m.out_pad * s->members * sizeof(float)) || !s->cnt.reserve(16 * sizeof(unsigned long long)))
    return set_error(TNG_ERR_CUDA, "tng_surrogate_predict: scratch allocation failed");
  int rc = solver_prepare(h);
  if (rc) return rc;
  unsigned long long* cnt = (unsigned long long*)s->cnt.ptr;
  cudaMemsetAsync(cnt, 0, 16 * sizeof(unsigned long long), st);
  rc = launch_infer(h, s, state, ncells, ld, dts, dt, p, 0, s->members, (float*)s->out.ptr, true, (int*)(cnt + 8));
  if (rc) return rc;
  SurPost pa = post_args(h, s, const_cast<double*>(state), ld, ncells, dts, dt, p);
  pa.out_state = out;
  pa.ld_out = ld_out;
  pa.reason_out = reason;
  pa.ind_out = indicator;
  k_sur_post<<<(int)std::min<int64_t>(4096, (ncells + 127) / 128), 128, 0, st>>>(pa);
  unsigned long long flag = 0;
  cudaMemcpyAsync(&flag, cnt + 8, sizeof(flag), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_error(e, "tng_surrogate_predict");
  if (flag) return set_error(TNG_ERR_CUDA, "tng_surrogate_predict: tensor-core inference timed out");
  return TNG_OK;
}

}  // extern "C"
