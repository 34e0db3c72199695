// The per-cell BDF integration (warp-cooperative) and the persistent work-stealing kernel.
// Same algorithm and constants as oracle/solver_oracle.c (orc_bdf_cell).
#pragma once
#include "solver.cuh"

namespace tng {

struct BdfCoef {
  double L[kQmax + 2][kQmax + 2];
  double errc[kQmax + 2], dnc[kQmax + 2], upc[kQmax + 2];
  // grow[e]: (2/3)^e (1 + 1e-9). For x > grow[e], x^(1/e) > 2/3 with a margin far above the
  // rounding of the power, so the step-size candidate 1 / (x^(1/e) + 1e-6) is below 1.5
  double grow[kQmax + 3];
};

struct BdfLaunch {
  BdfArgs a;
  const BdfCoef* coef;  // device copy of the BDF coefficients (staged into shared memory per block)
  const int* n_in_dev;  // when non-null, the number of queued cells is read from device memory
  int cold_in_smem;     // the Jacobian's term lists staged in shared memory (after the hot tables)
};

// two-entry-per-lane vector helpers (the weighted RMS norm out of line: it is evaluated at six
// places of the step and each inlined copy carried its own square root and division)
static __device__ __noinline__ double wrms2(const double v0, const double v1, const double w0, const double w1,
                                        const int nv, const int lane) {
  const double a = lane < nv ? v0 * w0 : 0.0;
  const double b = lane + 32 < nv ? v1 * w1 : 0.0;
  return sqrt(warp_sum(a * a + b * b) / nv);
}

__device__ __forceinline__ bool warp_all_finite(const double v0, const double v1, const int nv, const int lane) {
  const bool ok = (lane >= nv || isfinite(v0)) && (lane + 32 >= nv || isfinite(v1));
  return __all_sync(kFull, ok);
}

#define TNG_ZLOOP(j) _Pragma("unroll") for (int j = 0; j <= kQmax + 1; ++j)

// The Newton loop's two threshold tests, decided without their division unless the operands lie
// within a relative 1e-12 of the threshold (the rounding of the quotient is far smaller, so the
// outcome is that of the test on the rounded quotient; NaN operands take the division):
//  * |gamma / gamma_lu - 1| > dgmax (gamma_lu > 0: a factorisation exists when this is asked);
__device__ __forceinline__ bool gamma_moved(const double gamma, const double gamma_lu, const double dgmax) {
  const double up = gamma_lu * (1.0 + dgmax), dn = gamma_lu * (1.0 - dgmax);
  if (gamma > up * (1.0 + 1e-12) || gamma < dn * (1.0 - 1e-12)) return true;
  if (gamma < up * (1.0 - 1e-12) && gamma > dn * (1.0 + 1e-12)) return false;
  return fabs(div_ool(gamma, gamma_lu) - 1.0) > dgmax;
}
//  * the convergence test x / 0.1 <= 1.
__device__ __forceinline__ bool below_tenth(const double x) {
  if (x < 0.1 * (1.0 - 1e-12)) return true;
  if (x > 0.1 * (1.0 + 1e-12)) return false;
  return div_ool(x, 0.1) <= 1.0;
}

// x^y of the step-size and order selection (x >= 0, 0 < y < 1), one out-of-line copy, as
// exp(y ln x) through the solver's own exp and log: these are step-size heuristics, and the
// library pow (an extended-precision logarithm) cost 3 % of the solver's time
static __device__ __noinline__ double bdf_pow(const double x, const double y) { return exp_ool(y * log_ool(x)); }

__device__ __forceinline__ void z_predict(double (&z)[kQmax + 2][2], const int q) {
#pragma unroll
  for (int k = 0; k < kQmax; ++k) {
    if (k < q) {
#pragma unroll
      for (int j = kQmax; j > 0; --j)
        if (j > k && j <= q) {
          z[j - 1][0] += z[j][0];
          z[j - 1][1] += z[j][1];
        }
    }
  }
}

__device__ __forceinline__ void z_retract(double (&z)[kQmax + 2][2], const int q) {
#pragma unroll
  for (int k = kQmax - 1; k >= 0; --k) {
    if (k < q) {
#pragma unroll
      for (int j = 1; j <= kQmax; ++j)
        if (j > k && j <= q) {
          z[j - 1][0] -= z[j][0];
          z[j - 1][1] -= z[j][1];
        }
    }
  }
}

__device__ __forceinline__ void z_rescale(double (&z)[kQmax + 2][2], const int q, const double eta) {
  double f = 1.0;
#pragma unroll
  for (int j = 1; j <= kQmax + 1; ++j) {
    f *= eta;
    if (j <= q) {
      z[j][0] *= f;
      z[j][1] *= f;
    }
  }
}

__device__ __forceinline__ double zget(const double (&z)[kQmax + 2][2], const int j, const int h) {
  double v = 0.0;
#pragma unroll
  for (int k = 0; k <= kQmax + 1; ++k)
    if (k == j) v = z[k][h];
  return v;
}

__device__ __forceinline__ void zset(double (&z)[kQmax + 2][2], const int j, const int h, const double v) {
#pragma unroll
  for (int k = 0; k <= kQmax + 1; ++k)
    if (k == j) z[k][h] = v;
}

// Initial step size from an estimate of ||y''|| at the cell's initial state u (f = rhs(u), ew the
// error weights), at most dt. One out-of-line copy: it runs once per cell, and inlined (its loop
// unrolled) it made up a tenth of the solver's code.
template <class LY>
static __device__ __noinline__ double bdf_initial_step(const SvT<LY> t, double* wb, const double u0, const double u1,
                                                       const double f0, const double f1, const double ew0,
                                                       const double ew1, const double dt, const double atol,
                                                       const double p, const int lane) {
  constexpr int nv = SvT<LY>::NV;
  const bool h0 = lane < nv, h1 = lane + 32 < nv;
  const double hlb = 100.0 * 2.220446049250313e-16 * dt;
  double hub = 0.1 * dt;
  double r = 0.0;
  if (h0) r = fabs(f0) / (0.1 * fabs(u0) + atol);
  if (h1) r = fmax(r, fabs(f1) / (0.1 * fabs(u1) + atol));
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_xor_sync(kFull, r, off));
  if (hub * r > 1.0) hub = 1.0 / r;
  double hg = sqrt(hlb * hub), hnew = hg;
  if (hub < hlb) {
    hnew = hlb;
  } else {
#pragma unroll 1
    for (int it = 0; it < 4; ++it) {
      const double2 gg = rhs_call(t, wb, u0 + hg * f0, u1 + hg * f1, p, lane);
      const double ydd = wrms2((gg.x - f0) / hg, (gg.y - f1) / hg, ew0, ew1, nv, lane);
      hnew = (ydd * hub * hub > 2.0) ? sqrt(2.0 / ydd) : sqrt(hg * hub);
      if (!isfinite(hnew)) hnew = hg;
      const double hrat = hnew / hg;
      if (it == 3 || (hrat > 0.5 && hrat < 2.0)) break;
      hg = hnew;
    }
    hnew *= 0.5;
    if (hnew < hlb) hnew = hlb;
    if (hnew > hub) hnew = hub;
  }
  return hnew < dt ? hnew : dt;
}

// Integrate one cell (warp-cooperative). Returns true when the cell is finished (any status),
// false when it used up the pass budget and was saved for the next pass.
template <class LY>
__device__ __forceinline__ bool bdf_cell(const BdfLaunch& P, const BdfCoef& C, const SvT<LY>& t, const WarpMem& w,
                                         const int cell, const int lane) {
  const BdfArgs& a = P.a;
  constexpr int ns = SvT<LY>::NS, nv = ns + 1, rs = SvT<LY>::RS;
  const double dt = a.dts ? a.dts[cell] : a.dt_scalar;
  const double p = a.p, rtol = a.rtol, atol = a.atol;
  const bool h0 = lane < nv, h1 = lane + 32 < nv;
  double z[kQmax + 2][2];
  double acorp[2] = {0.0, 0.0}, ewt[2] = {0.0, 0.0}, acor[2], y[2], f[2], x[2];
  TNG_ZLOOP(j) { z[j][0] = 0.0; z[j][1] = 0.0; }
  double tcur = 0.0, h = 0.0, hprev = 0.0, crate = 1.0, etamax = 1e4, gamma_lu = 0.0;
  int q = 1, qwait = 2, qprev = 0, need_j = 1, nst_lu = 0, nst = 0, nni = 0, nje = 0, status = ST_OK;
  double* sv = a.save ? a.save + (long long)cell * a.save_stride : nullptr;
  const bool resume = a.resume && a.resume[cell];
  if (resume) {
    TNG_ZLOOP(j) {
      if (j <= kQmax) {
        z[j][0] = h0 ? sv[j * nv + lane] : 0.0;
        z[j][1] = h1 ? sv[j * nv + lane + 32] : 0.0;
      }
    }
    acorp[0] = h0 ? sv[(kQmax + 1) * nv + lane] : 0.0;
    acorp[1] = h1 ? sv[(kQmax + 1) * nv + lane + 32] : 0.0;
    const double* s = sv + (kQmax + 2) * nv;
    tcur = s[0], h = s[1], hprev = s[2], crate = s[3], etamax = s[4];
    q = (int)s[5], qwait = (int)s[6], qprev = (int)s[7], nst = (int)s[8], nni = (int)s[9], nje = (int)s[10];
    need_j = 1;
    nst_lu = nst;
    ewt[0] = h0 ? div_ool(1.0, rtol * fabs(z[0][0]) + atol) : 0.0;
    ewt[1] = h1 ? div_ool(1.0, rtol * fabs(z[0][1]) + atol) : 0.0;
  } else {
    const long long ld = a.ld;
    const double u0 = h0 ? a.state[(long long)lane * ld + cell] : 0.0;
    const double u1 = h1 ? a.state[(long long)(lane + 32) * ld + cell] : 0.0;
    z[0][0] = u0;
    z[0][1] = u1;
    if (!(dt > 0.0)) goto finish;
    ewt[0] = h0 ? div_ool(1.0, rtol * fabs(u0) + atol) : 0.0;
    ewt[1] = h1 ? div_ool(1.0, rtol * fabs(u1) + atol) : 0.0;
    {
      const double2 r = rhs_call(t, w.mat, u0, u1, p, lane);
      f[0] = r.x, f[1] = r.y;
    }
    if (!warp_all_finite(f[0], f[1], nv, lane)) {
      status = ST_NONFINITE;
      goto finish;
    }
    h = bdf_initial_step<LY>(t, w.mat, u0, u1, f[0], f[1], ewt[0], ewt[1], dt, atol, p, lane);
    z[1][0] = h * f[0];
    z[1][1] = h * f[1];
    hprev = h;
  }
  {
    const double hlb = 100.0 * 2.220446049250313e-16 * dt;
    const int maxcor = a.maxcor > 0 ? a.maxcor : 3;
    const int msbp = a.msbp > 0 ? a.msbp : 20;
    const double dgmax = a.dgmax > 0.0 ? a.dgmax : 0.3;
    int pass_steps = 0;
    while (tcur < dt) {
      if (nst >= a.max_steps) {
        status = ST_MAXSTEPS;
        break;
      }
      if (pass_steps >= a.budget) {
        // save the history for the next pass and queue the cell again
        TNG_ZLOOP(j) {
          if (j <= kQmax) {
            if (h0) sv[j * nv + lane] = z[j][0];
            if (h1) sv[j * nv + lane + 32] = z[j][1];
          }
        }
        if (h0) sv[(kQmax + 1) * nv + lane] = acorp[0];
        if (h1) sv[(kQmax + 1) * nv + lane + 32] = acorp[1];
        if (lane == 0) {
          double* s = sv + (kQmax + 2) * nv;
          s[0] = tcur, s[1] = h, s[2] = hprev, s[3] = crate, s[4] = etamax;
          s[5] = q, s[6] = qwait, s[7] = qprev, s[8] = nst, s[9] = nni, s[10] = nje;
          a.resume[cell] = 1;
          const int slot = atomicAdd(a.n_out, 1);
          a.queue_out[slot] = cell;
        }
        __syncwarp();
        return false;
      }
      if (tcur + h > dt) {
        const double eta = div_ool(dt - tcur, h);
        z_rescale(z, q, eta);
        h = dt - tcur;
      }
      int ncf = 0, nef = 0;
      double dsm = 0.0;
      bool fail = false;
      for (;;) {  // attempt the step
        if (h < hlb * 1e-3 || !isfinite(h)) {
          status = ST_HMIN;
          fail = true;
          break;
        }
        z_predict(z, q);
        const double l0 = C.L[q][0];
        const double gamma = h * l0;
        bool conv_fail = false;
        bool jcur = false;
        if (need_j || nst >= nst_lu + msbp || gamma_moved(gamma, gamma_lu, dgmax)) {
          {
            const double2 r = rhs_call(t, w.mat, z[0][0], z[0][1], p, lane, 1);  // keeps the rate constants
            f[0] = r.x, f[1] = r.y;
          }
          jac_call(t, w.mat, z[0][0], z[0][1], f[0], f[1], p, lane);
          ++nje;
#pragma unroll 4
          for (int e = lane; e < nv * rs; e += 32) w.mat[e] = -gamma * w.mat[e];
          __syncwarp();
          for (int i = lane; i < nv; i += 32) w.mat[i * rs + i] += 1.0;
          __syncwarp();
          const int sing = lu_call<LY>(w.mat, lane);
          gamma_lu = gamma;
          nst_lu = nst;
          jcur = true;
          need_j = 0;
          crate = 1.0;
          if (sing) conv_fail = true;
        }
        if (!conv_fail) {
          double delp = 0.0;
          // correction scale for a factorisation made at another gamma (fixed over the attempt)
          const double cf = gamma != gamma_lu ? div_ool(2.0, 1.0 + div_ool(gamma, gamma_lu)) : 1.0;
          acor[0] = acor[1] = 0.0;
          y[0] = z[0][0];
          y[1] = z[0][1];
          conv_fail = true;
#pragma unroll 1
          for (int it = 0; it < maxcor; ++it) {
            // the first iterate is the predicted state: after a new Jacobian, f already holds
            // the right-hand side there (the Jacobian was formed around it)
            if (it > 0 || !jcur) {
              const double2 r = rhs_call(t, w.mat, y[0], y[1], p, lane);
              f[0] = r.x, f[1] = r.y;
            }
            ++nni;
            x[0] = h * f[0] - z[1][0] - acor[0];
            x[1] = h * f[1] - z[1][1] - acor[1];
            lu_solve_reg(w.mat, nv, rs, w.perm, w.cb, w.vb, x[0], x[1], lane);
            if (!h0) x[0] = 0.0;
            if (!h1) x[1] = 0.0;
            if (gamma != gamma_lu) {
              x[0] *= cf;
              x[1] *= cf;
            }
            acor[0] += x[0];
            acor[1] += x[1];
            y[0] = z[0][0] + l0 * acor[0];
            y[1] = z[0][1] + l0 * acor[1];
            const double del = wrms2(x[0], x[1], ewt[0], ewt[1], nv, lane);
            if (!isfinite(del)) break;
            if (it > 0) crate = fmax(0.3 * crate, div_ool(del, delp));
            if (below_tenth(del * fmin(1.0, crate) * C.errc[q])) {
              conv_fail = false;
              break;
            }
            if (it > 0 && del > 2.0 * delp) break;
            delp = del;
          }
        }
        if (conv_fail) {
          z_retract(z, q);
          ++ncf;
          if (ncf >= 10) {
            status = ST_CONVFAIL;
            fail = true;
            break;
          }
          if (!jcur) {
            need_j = 1;
            continue;
          }
          z_rescale(z, q, 0.25);
          h *= 0.25;
          need_j = 1;
          continue;
        }
        dsm = C.errc[q] * wrms2(acor[0], acor[1], ewt[0], ewt[1], nv, lane);
        if (dsm > 1.0) {
          z_retract(z, q);
          ++nef;
          if (nef >= 7) {
            status = ST_ERRFAIL;
            fail = true;
            break;
          }
          if (nef >= 3 && q > 1) {
            h *= 0.1;
            q = 1;
            {
              const double2 r = rhs_call(t, w.mat, z[0][0], z[0][1], p, lane);
              f[0] = r.x, f[1] = r.y;
            }
            z[1][0] = h * f[0];
            z[1][1] = h * f[1];
            qwait = 2;
            qprev = 0;
            continue;
          }
          double eta = div_ool(1.0, bdf_pow(6.0 * dsm, div_ool(1.0, q + 1)) + 1e-6);
          eta = fmax(0.1, fmin(0.9, eta));
          if (nef >= 2) eta = fmin(eta, 0.2);
          z_rescale(z, q, eta);
          h *= eta;
          continue;
        }
        break;
      }
      if (fail) break;
      // accept
      tcur += h;
      ++nst;
      ++pass_steps;
#pragma unroll
      for (int j = 0; j <= kQmax; ++j)
        if (j <= q) {
          z[j][0] += C.L[q][j] * acor[0];
          z[j][1] += C.L[q][j] * acor[1];
        }
      if (!warp_all_finite(z[0][0], z[0][1], nv, lane)) {
        status = ST_NONFINITE;
        break;
      }
      {
        const double e0 = div_ool(1.0, rtol * fabs(z[0][0]) + atol);
        const double e1 = div_ool(1.0, rtol * fabs(z[0][1]) + atol);
        ewt[0] = h0 ? e0 : 0.0;
        ewt[1] = h1 ? e1 : 0.0;
      }
      if (tcur >= dt) break;
      --qwait;
      // A candidate below 1.5 never decides the outcome (a larger one wins, or all are below 1.5
      // and the step is kept), so its power is skipped where the argument shows it is below 1.5.
      const double eta_q =
          6.0 * dsm > C.grow[q + 1] ? 0.0 : div_ool(1.0, bdf_pow(6.0 * dsm, div_ool(1.0, q + 1)) + 1e-6);
      double eta_m = 0.0, eta_p = 0.0;
      if (qwait <= 0) {
        if (q > 1) {
          const double ddn = C.dnc[q] * wrms2(zget(z, q, 0), zget(z, q, 1), ewt[0], ewt[1], nv, lane);
          eta_m = 6.0 * ddn > C.grow[q] ? 0.0 : div_ool(1.0, bdf_pow(6.0 * ddn, div_ool(1.0, q)) + 1e-6);
        }
        if (q < kQmax && qprev == q) {
          double r = div_ool(h, hprev);  // (h / hprev)^(q + 1)
          {
            const double b = r;
            for (int i = 1; i <= q; ++i) r *= b;
          }
          const double dup =
              C.upc[q] * wrms2(acor[0] - r * acorp[0], acor[1] - r * acorp[1], ewt[0], ewt[1], nv, lane);
          eta_p = 10.0 * dup > C.grow[q + 2] ? 0.0 : div_ool(1.0, bdf_pow(10.0 * dup, div_ool(1.0, q + 2)) + 1e-6);
        }
      }
      double eta = eta_q;
      int newq = q;
      if (eta_m > eta) {
        eta = eta_m;
        newq = q - 1;
      }
      if (eta_p > eta) {
        eta = eta_p;
        newq = q + 1;
      }
      if (eta < 1.5) {
        eta = 1.0;
        newq = q;
      } else if (eta > etamax) {
        eta = etamax;
      }
      etamax = 10.0;
      acorp[0] = acor[0];
      acorp[1] = acor[1];
      qprev = q;
      hprev = h;
      if (newq == q + 1) {
        const double c = div_ool(C.L[q][q], q + 1);
        zset(z, q + 1, 0, c * acor[0]);
        zset(z, q + 1, 1, c * acor[1]);
        q = q + 1;
        qprev = 0;
      } else if (newq == q - 1) {
        q = q - 1;
        qprev = 0;
      }
      if (eta != 1.0 || qprev == 0)
        qwait = q + 1;
      else if (qwait <= 0)
        qwait = 2;
      if (eta != 1.0) {
        z_rescale(z, q, eta);
        h *= eta;
      }
    }
  }
finish:
  {
    const long long ld = a.ld;
    if (h0) a.state[(long long)lane * ld + cell] = z[0][0];
    if (h1) a.state[(long long)(lane + 32) * ld + cell] = z[0][1];
    if (lane == 0) {
      if (a.nst) a.nst[cell] = nst;
      if (a.nni) a.nni[cell] = nni;
      if (a.nje) a.nje[cell] = nje;
      if (a.status) a.status[cell] = status;
      if (a.resume) a.resume[cell] = 0;
    }
    __syncwarp();
  }
  return true;
}

// Shared memory of one block: the staged hot tables, then one workspace per warp.
__host__ __device__ inline int hot_smem_doubles(const SvLayout& L) { return (hot_smem_bytes(L) + 15) / 16 * 2; }

// BDF coefficients (l-vectors per order, error constants) as the host computes them.
BdfCoef make_coef();

// One block per SM of WARPS warps (the staged tables are shared by the block's warps),
// specialised on the mechanism's layout LY; instantiated once per mechanism (generated unit).
template <class LY, int WARPS, int MINB = 1>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_bdf(const BdfLaunch P) {
  extern __shared__ __align__(16) double smem[];
  __shared__ BdfCoef s_coef;
  {
    const double* src = reinterpret_cast<const double*>(P.coef);
    double* dst = reinterpret_cast<double*>(&s_coef);
    for (int e = threadIdx.x; e < (int)(sizeof(BdfCoef) / sizeof(double)); e += blockDim.x) dst[e] = src[e];
  }
  SvT<LY> t = stage_tables<LY>(P.a.tab, smem);  // synchronises the block
  size_t off = hot_smem_doubles(P.a.tab.L);
  if (P.cold_in_smem) {
    t = stage_cold_tables<LY>(t, smem + off);
    off += cold_smem_doubles(P.a.tab.L);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpMem w = warp_mem<LY>(smem + off + (size_t)warp * P.a.smem_warp);
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.a.n_in;
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(P.a.head, 1);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= n_in) break;
    const int cell = P.a.queue_in ? P.a.queue_in[idx] : idx;
    bdf_cell<LY>(P, s_coef, t, w, cell, lane);
  }
}

// Standalone right-hand side / Jacobian of the table-driven warp path (parity checks).
template <class LY, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    k_warp_rhs_jac(SvDev g, const double* __restrict__ state, long long ld, int n, double p, double* __restrict__ rhs,
                   double* __restrict__ jac, int smem_warp) {
  extern __shared__ __align__(16) double smem[];
  const SvT<LY> t = stage_tables<LY>(g, smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpMem w = warp_mem<LY>(smem + hot_smem_doubles(g.L) + (size_t)warp * smem_warp);
  constexpr int nv = SvT<LY>::NV, rs = SvT<LY>::RS;
  for (int cell = blockIdx.x * WARPS + warp; cell < n; cell += gridDim.x * WARPS) {
    const double y0 = lane < nv ? state[(long long)lane * ld + cell] : 0.0;
    const double y1 = lane + 32 < nv ? state[(long long)(lane + 32) * ld + cell] : 0.0;
    const double2 r = rhs_call(t, w.mat, y0, y1, p, lane, jac != nullptr);  // keeps the rate constants
    const double f0 = r.x, f1 = r.y;
    if (lane < nv) rhs[(long long)lane * ld + cell] = f0;
    if (lane + 32 < nv) rhs[(long long)(lane + 32) * ld + cell] = f1;
    if (jac) {
      jac_call(t, w.mat, y0, y1, f0, f1, p, lane);
      for (int e = lane; e < nv * nv; e += 32) jac[(long long)cell * nv * nv + e] = w.mat[(e / nv) * rs + e % nv];
      __syncwarp();
    }
  }
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes`, never lower it: the batch
// solver and the no-allocation entry launch the same kernels with different shared-memory
// plans, and each must keep working after the other has run.
inline cudaError_t ensure_dynamic_smem(const void* kernel, size_t bytes) {
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// The solver kernels of one mechanism (instantiated in the mechanism's generated unit and
// reached through its operation table): two sets, [0] with FP64 rate-constant exponentials and
// [1] with the mixed form (solver_kernels_for picks by the handle's precision).
typedef void (*BdfKernelFn)(const BdfLaunch);
typedef void (*RhsJacFn)(SvDev, const double*, long long, int, double, double*, double*, int);
struct SolverKernels {
  BdfKernelFn bdf2, bdf4, bdf8, bdf8_occ2;  // warps per block; bdf8_occ2: two blocks per SM (128 registers)
  RhsJacFn rhs_jac4;
};

template <class LX>
constexpr SolverKernels solver_kernel_set() {
  return {k_bdf<LX, 2>, k_bdf<LX, 4>, k_bdf<LX, 8>, k_bdf<LX, 8, 2>, k_warp_rhs_jac<LX, 4>};
}

template <class LY>
const SolverKernels* solver_kernels() {
  static const SolverKernels k[2] = {solver_kernel_set<SvLX<LY, 0>>(), solver_kernel_set<SvLX<LY, 1>>()};
  return k;
}

// The kernel set for a precision flag (SvDev::mixed).
inline const SolverKernels* solver_kernels_for(const SolverKernels* sets, const int mixed) {
  return sets + (mixed ? 1 : 0);
}

static __global__ void k_reset_counters(int* a, int* b) {
  if (threadIdx.x == 0) {
    *a = 0;
    if (b) *b = 0;
  }
}

}  // namespace tng
