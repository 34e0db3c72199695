/* CPU restatement of the implicit chemistry substep -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load this; the product never
 * links it. It is the CPU twin of the GPU solver (tiger_nga_b200/csrc/solver.cu): same
 * Jacobian, same LU, same integrator and step control, so that the two can be compared cell
 * by cell, and it is the timed CPU baseline of the substep (OpenMP over cells, the analogue of
 * the reference's one MPI rank per core).
 *
 * What it replaces in the reference: finitechem_source_chemistry (combustion/finitechem.f90:
 * 962-1071) integrates each cell with SUNDIALS CVODE 2.5.0 (external, not vendored; called at
 * finitechem.f90:987-1068): BDF orders 1-5, Newton iteration with a dense direct solver and a
 * difference-quotient Jacobian, rtol 1e-6 / atol 1e-12 (finitechem.f90:266-267), at most
 * 10000 steps (:1025), stopping exactly at dt (:1022). This restates that published method:
 *   - variable-order (1..5), variable-step BDF in Nordsieck form; a step change rescales the
 *     history (z_j *= eta^j); the corrector vector of order q is the coefficient list of
 *     prod_{i=1..q} (1 + x/i), normalised so that l_1 = 1;
 *   - modified Newton on M = I - gamma J, gamma = h l_0; J and its LU are refreshed when stale
 *     (first step, convergence failure, every 20 steps, or gamma moved by more than 30%);
 *     convergence when ||dx|| min(1, rate) <= 0.1 / E_q (E_q the error-test constant);
 *   - local error E_q ||acor||_WRMS <= 1 with weights 1/(rtol |y| + atol); order selection
 *     among q-1, q, q+1 with bias factors 6, 6, 10; step growth capped at 10 (10^4 after the
 *     first step); failure handling with factors 0.25 (convergence) and 0.1..0.9 (error);
 *   - the initial step from an estimate of ||y''|| (two to four right-hand sides);
 *   - the Jacobian is analytic in the species columns (mass action, third bodies, falloff
 *     through [M] at fixed broadening) and a forward difference in the temperature column; the
 *     temperature row follows from the species rows (finitechem.f90:160-173 differentiated).
 * CVODE's own source is absent, so the integrator's parity with the reference is unpinned:
 * it is checked against a tight-tolerance independent integration instead.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "orc_mech.h"

void orc_rhs(const orc_mech *m, const double *sol, double p, double *rhs);
void orc_prodrates(const orc_mech *m, double *cdot, double *W, double *K, const double *C, double *M, double T,
                   double P);
void orc_thermo(const orc_mech *m, double T, double *h, double *cp);

#define MAXV 64
#define MAXR 1024
#define QMAX 5

typedef struct {
  double rtol, atol;
  int max_steps, maxcor, msbp;
  double dgmax;
} orc_solver_cfg;

typedef struct {
  int status; /* 0 ok, 1 max steps, 2 convergence failures, 3 error-test failures, 4 non-finite, 5 h underflow */
  int nst, nni, nje, nef, ncf, nrhs, q;
  double h;
} orc_cell_stats;

/* ------------------------------------------------------------------------------------- */
/* Jacobian of finitechem_compute_rhs w.r.t. the state (rho*Y_1..N, rho*T), row-major NVxNV */

static double arrh_v(int flags, double A, double n, double E, double LT, double RT) {
  if (!(flags & 6)) return A;
  double arg;
  if ((flags & 2) && (flags & 4))
    arg = n * LT + E / RT;
  else if (flags & 2)
    arg = n * LT;
  else
    arg = E / RT;
  return A * exp(arg);
}

void orc_jacobian(const orc_mech *m, const double *u, double p, const double *f0, double *J) {
  const int N = m->ns, NV = N + 1;
  double C[MAXV], Mtb[MAXV], K[MAXR], W[MAXR], cd[MAXV], h[MAXV], cp[MAXV];
  static __thread double A[MAXV * MAXV], G[MAXV * MAXV];
  double rho = 0.0;
  for (int k = 0; k < N; ++k) rho += u[k];
  const double T = u[N] / rho;
  for (int k = 0; k < N; ++k) C[k] = u[k] / m->wmol[k];
  orc_prodrates(m, cd, W, K, C, Mtb, T, p);
  memset(A, 0, sizeof(double) * N * N);
  memset(G, 0, sizeof(double) * N * (m->nm > 0 ? m->nm : 1));
  const double LT = log(T), RT = m->rgas * T;
  for (int r = 0; r < m->nslot; ++r) {
    const int b = m->w_ptr[r], e = m->w_ptr[r + 1];
    const double mfac = m->w_M[r] >= 0 ? Mtb[m->w_M[r]] : 1.0;
    double prodC = 1.0;
    for (int i = b; i < e; ++i) prodC *= C[m->w_sp[i]];
    for (int pidx = b; pidx < e; ++pidx) {
      double d = K[r] * mfac;
      for (int i = b; i < e; ++i)
        if (i != pidx) d *= C[m->w_sp[i]];
      const int j = m->w_sp[pidx];
      for (int i = 0; i < N; ++i) {
        const double nu = m->nu[i * m->nslot + r];
        if (nu != 0.0) A[i * N + j] += nu * d;
      }
    }
    if (m->w_M[r] >= 0) {
      const double g = K[r] * prodC;
      for (int i = 0; i < N; ++i) {
        const double nu = m->nu[i * m->nslot + r];
        if (nu != 0.0) G[i * m->nm + m->w_M[r]] += nu * g;
      }
    }
    if (m->k_flags[r] & 1) {
      const int f = m->k_fo[r];
      const double Mf = Mtb[m->fo_M[f]];
      if (Mf > 0.0) {
        const double k0 = arrh_v(m->f0_flags[f], m->f0A[f], m->f0n[f], m->f0E[f], LT, RT);
        const double ki = arrh_v(m->fi_flags[f], m->fiA[f], m->fin[f], m->fiE[f], LT, RT);
        const double pr = k0 * Mf / fmax(ki, m->troe[5]);
        const double g = K[r] / (Mf * (1.0 + pr)) * prodC * mfac;
        for (int i = 0; i < N; ++i) {
          const double nu = m->nu[i * m->nslot + r];
          if (nu != 0.0) G[i * m->nm + m->fo_M[f]] += nu * g;
        }
      }
    }
  }
  for (int i = 0; i < N; ++i)
    for (int mm = 0; mm < m->nm; ++mm) {
      const double g = G[i * m->nm + mm];
      if (g == 0.0) continue;
      for (int j = 0; j < N; ++j) A[i * N + j] += g * m->eff[mm * N + j];
    }
  /* temperature column: forward difference */
  double u1[MAXV], f1[MAXV];
  for (int v = 0; v < NV; ++v) u1[v] = u[v];
  const double dlt = sqrt(DBL_EPSILON) * fmax(fabs(u[N]), 1e-30);
  u1[N] = u[N] + dlt;
  orc_rhs(m, u1, p, f1);
  const double idl = 1.0 / (u1[N] - u[N]);
  for (int i = 0; i < NV; ++i) J[i * NV + N] = (f1[i] - f0[i]) * idl;
  /* species columns */
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) J[i * NV + j] = m->wmol[i] * A[i * N + j] / m->wmol[j] - T * J[i * NV + N];
  /* temperature row */
  orc_thermo(m, T, h, cp);
  const double *tab = (T > m->tmid) ? m->th_hi : m->th_lo;
  double cpm = 0.0, scp = 0.0, ydcp = 0.0;
  for (int k = 0; k < N; ++k) {
    const double *t = tab + 12 * k;
    const double dcp = t[0] * (t[8] + T * (2.0 * t[9] + T * (3.0 * t[10] + T * (4.0 * t[11]))));
    const double y = u[k] / rho;
    cpm += y * cp[k];
    ydcp += y * dcp;
    scp += cp[k] * f0[k];
  }
  const double dTdu = -T / rho;
  for (int j = 0; j < N; ++j) {
    double s = 0.0;
    for (int k = 0; k < N; ++k) s += h[k] * J[k * NV + j];
    s += dTdu * scp;
    const double dcpm = (cp[j] - cpm) / rho + dTdu * ydcp;
    J[N * NV + j] = -(s + f0[N] * dcpm) / cpm;
  }
}

/* ------------------------------------------------------------------------------------- */
/* LU with partial pivoting (first maximum), row-major, in place; returns 0 or 1 if singular */

int orc_lu(double *A, int n, int *piv) {
  int sing = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(A[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = fabs(A[i * n + k]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        const double t = A[k * n + j];
        A[k * n + j] = A[p * n + j];
        A[p * n + j] = t;
      }
    const double d = A[k * n + k];
    if (d == 0.0) {
      sing = 1;
      continue;
    }
    for (int i = k + 1; i < n; ++i) A[i * n + k] = A[i * n + k] / d;
    for (int i = k + 1; i < n; ++i) {
      const double l = A[i * n + k];
      for (int j = k + 1; j < n; ++j) A[i * n + j] = fma(-l, A[k * n + j], A[i * n + j]);
    }
  }
  return sing;
}

void orc_lu_solve(const double *A, int n, const int *piv, double *b) {
  for (int k = 0; k < n; ++k) {
    const int p = piv[k];
    if (p != k) {
      const double t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
  for (int k = 0; k < n; ++k)
    for (int i = k + 1; i < n; ++i) b[i] = fma(-A[i * n + k], b[k], b[i]);
  for (int k = n - 1; k >= 0; --k) {
    b[k] = b[k] / A[k * n + k];
    for (int i = 0; i < k; ++i) b[i] = fma(-A[i * n + k], b[k], b[i]);
  }
}

/* ------------------------------------------------------------------------------------- */
/* BDF integrator */

static double L[QMAX + 2][QMAX + 2];
static double ERRC[QMAX + 2], DNC[QMAX + 2], UPC[QMAX + 2];
static int coef_ready = 0;

static void bdf_coefficients(void) {
  /* l(x) = prod_{i=1..q} (1 + x/i), normalised to l_1 = 1 */
  for (int q = 1; q <= QMAX + 1; ++q) {
    double c[QMAX + 3] = {1.0};
    for (int i = 1; i <= q; ++i)
      for (int j = i; j >= 1; --j) c[j] += c[j - 1] / (double)i;
    for (int j = 0; j <= q; ++j) L[q][j] = c[j] / c[1];
  }
  double fact = 1.0;
  for (int q = 1; q <= QMAX; ++q) {
    fact *= q;
    ERRC[q] = L[q][0] / (q + 1) * fact * L[q][q];      /* LTE of order q from acor */
    DNC[q] = q > 1 ? L[q - 1][0] / q * fact : 0.0;     /* LTE of order q-1 from z_q */
    UPC[q] = L[q + 1][0] / (q + 2) * fact * L[q][q];   /* LTE of order q+1 from acor differences */
  }
  coef_ready = 1;
}

void orc_bdf_constants(double *l_out, double *errc, double *dnc, double *upc) {
  if (!coef_ready) bdf_coefficients();
  for (int q = 0; q <= QMAX + 1; ++q)
    for (int j = 0; j <= QMAX + 1; ++j) l_out[q * (QMAX + 2) + j] = L[q][j];
  for (int q = 0; q <= QMAX + 1; ++q) {
    errc[q] = ERRC[q];
    dnc[q] = DNC[q];
    upc[q] = UPC[q];
  }
}

static double wrms(const double *v, const double *w, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) {
    const double x = v[i] * w[i];
    s += x * x;
  }
  return sqrt(s / n);
}

static void predict(double z[][MAXV], int q, int nv) {
  for (int k = 0; k < q; ++k)
    for (int j = q; j > k; --j)
      for (int i = 0; i < nv; ++i) z[j - 1][i] += z[j][i];
}

static void retract(double z[][MAXV], int q, int nv) {
  for (int k = q - 1; k >= 0; --k)
    for (int j = k + 1; j <= q; ++j)
      for (int i = 0; i < nv; ++i) z[j - 1][i] -= z[j][i];
}

static void rescale(double z[][MAXV], int q, int nv, double eta) {
  double f = 1.0;
  for (int j = 1; j <= q; ++j) {
    f *= eta;
    for (int i = 0; i < nv; ++i) z[j][i] *= f;
  }
}

static void set_ewt(const double *y, double *w, int nv, double rtol, double atol) {
  for (int i = 0; i < nv; ++i) w[i] = 1.0 / (rtol * fabs(y[i]) + atol);
}

static int all_finite(const double *v, int n) {
  for (int i = 0; i < n; ++i)
    if (!isfinite(v[i])) return 0;
  return 1;
}

/* Integrate one cell: u (NV) is overwritten with the state at dt. */
void orc_bdf_cell(const orc_mech *m, const orc_solver_cfg *cfg, double *u, double dt, double p,
                  orc_cell_stats *st) {
  if (!coef_ready) bdf_coefficients();
  const int N = m->ns, NV = N + 1;
  double z[QMAX + 2][MAXV], acor[MAXV], acorp[MAXV], y[MAXV], f[MAXV], ewt[MAXV], x[MAXV], tmp[MAXV];
  static __thread double J[MAXV * MAXV], Mx[MAXV * MAXV];
  int piv[MAXV];
  memset(st, 0, sizeof(*st));
  if (!(dt > 0.0)) return;
  const double rtol = cfg->rtol, atol = cfg->atol;
  set_ewt(u, ewt, NV, rtol, atol);
  orc_rhs(m, u, p, f);
  st->nrhs++;
  if (!all_finite(f, NV)) {
    st->status = 4;
    return;
  }
  /* initial step */
  const double hlb = 100.0 * DBL_EPSILON * dt;
  double hub = 0.1 * dt, hinv = 0.0;
  for (int i = 0; i < NV; ++i) {
    const double r = fabs(f[i]) / (0.1 * fabs(u[i]) + atol);
    if (r > hinv) hinv = r;
  }
  if (hub * hinv > 1.0) hub = 1.0 / hinv;
  double hg = sqrt(hlb * hub), hnew = hg;
  if (hub < hlb) {
    hnew = hlb;
  } else {
    for (int it = 0; it < 4; ++it) {
      for (int i = 0; i < NV; ++i) y[i] = u[i] + hg * f[i];
      orc_rhs(m, y, p, tmp);
      st->nrhs++;
      for (int i = 0; i < NV; ++i) x[i] = (tmp[i] - f[i]) / hg;
      const double ydd = wrms(x, ewt, NV);
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
  double h = hnew < dt ? hnew : dt;
  for (int i = 0; i < NV; ++i) {
    z[0][i] = u[i];
    z[1][i] = h * f[i];
    acorp[i] = 0.0;
  }
  int q = 1, qwait = 2, qprev = 0, need_j = 1, nst_lu = 0, jcur = 0;
  double t = 0.0, gamma_lu = 0.0, crate = 1.0, hprev = h, etamax = 1e4;
  const int maxcor = cfg->maxcor > 0 ? cfg->maxcor : 3;
  const int msbp = cfg->msbp > 0 ? cfg->msbp : 20;
  const double dgmax = cfg->dgmax > 0 ? cfg->dgmax : 0.3;
  while (t < dt) {
    if (st->nst >= cfg->max_steps) {
      st->status = 1;
      break;
    }
    if (t + h > dt) {
      const double eta = (dt - t) / h;
      rescale(z, q, NV, eta);
      h = dt - t;
    }
    int ncf = 0, nef = 0;
    double dsm = 0.0;
    for (;;) { /* attempt the step */
      if (h < hlb * 1e-3 || !isfinite(h)) {
        st->status = 5;
        goto done;
      }
      predict(z, q, NV);
      const double gamma = h * L[q][0];
      /* Newton */
      int conv = 0;
      if (need_j || st->nst >= nst_lu + msbp || fabs(gamma / gamma_lu - 1.0) > dgmax) {
        orc_rhs(m, z[0], p, f);
        st->nrhs++;
        orc_jacobian(m, z[0], p, f, J);
        st->nje++;
        st->nrhs++;
        for (int i = 0; i < NV * NV; ++i) Mx[i] = -gamma * J[i];
        for (int i = 0; i < NV; ++i) Mx[i * NV + i] += 1.0;
        const int sing = orc_lu(Mx, NV, piv);
        gamma_lu = gamma;
        nst_lu = st->nst;
        jcur = 1;
        need_j = 0;
        crate = 1.0;
        if (sing) {
          conv = 1;
          goto newton_done;
        }
      } else {
        jcur = 0;
      }
      {
        double delp = 0.0;
        for (int i = 0; i < NV; ++i) {
          acor[i] = 0.0;
          y[i] = z[0][i];
        }
        conv = 1;
        for (int it = 0; it < maxcor; ++it) {
          orc_rhs(m, y, p, f);
          st->nrhs++;
          st->nni++;
          for (int i = 0; i < NV; ++i) x[i] = h * f[i] - z[1][i] - acor[i];
          orc_lu_solve(Mx, NV, piv, x);
          if (gamma != gamma_lu) {
            const double c = 2.0 / (1.0 + gamma / gamma_lu);
            for (int i = 0; i < NV; ++i) x[i] *= c;
          }
          for (int i = 0; i < NV; ++i) {
            acor[i] += x[i];
            y[i] = z[0][i] + L[q][0] * acor[i];
          }
          const double del = wrms(x, ewt, NV);
          if (!isfinite(del)) break;
          if (it > 0) crate = fmax(0.3 * crate, del / delp);
          const double dcon = del * fmin(1.0, crate) * ERRC[q] / 0.1;
          if (dcon <= 1.0) {
            conv = 0;
            break;
          }
          if (it > 0 && del > 2.0 * delp) break;
          delp = del;
        }
      }
    newton_done:
      if (conv) {
        retract(z, q, NV);
        ncf++;
        st->ncf++;
        if (ncf >= 10) {
          st->status = 2;
          goto done;
        }
        if (!jcur) {
          need_j = 1;
          continue;
        }
        rescale(z, q, NV, 0.25);
        h *= 0.25;
        need_j = 1;
        continue;
      }
      dsm = ERRC[q] * wrms(acor, ewt, NV);
      if (dsm > 1.0) {
        retract(z, q, NV);
        nef++;
        st->nef++;
        if (nef >= 7) {
          st->status = 3;
          goto done;
        }
        if (nef >= 3 && q > 1) {
          /* fall back to order 1, restart the history from f at the last accepted point */
          const double eta = 0.1;
          h *= eta;
          q = 1;
          orc_rhs(m, z[0], p, f);
          st->nrhs++;
          for (int i = 0; i < NV; ++i) z[1][i] = h * f[i];
          qwait = 2;
          qprev = 0;
          continue;
        }
        double eta = 1.0 / (pow(6.0 * dsm, 1.0 / (q + 1)) + 1e-6);
        eta = fmax(0.1, fmin(0.9, eta));
        if (nef >= 2) eta = fmin(eta, 0.2);
        rescale(z, q, NV, eta);
        h *= eta;
        continue;
      }
      break;
    }
    /* accept */
    t += h;
    st->nst++;
    for (int j = 0; j <= q; ++j)
      for (int i = 0; i < NV; ++i) z[j][i] += L[q][j] * acor[i];
    if (!all_finite(z[0], NV)) {
      st->status = 4;
      goto done;
    }
    set_ewt(z[0], ewt, NV, rtol, atol);
    if (t >= dt) break;
    /* step size and order for the next step */
    qwait--;
    const double eta_q = 1.0 / (pow(6.0 * dsm, 1.0 / (q + 1)) + 1e-6);
    double eta_m = 0.0, eta_p = 0.0;
    if (qwait <= 0) {
      if (q > 1) {
        const double ddn = DNC[q] * wrms(z[q], ewt, NV);
        eta_m = 1.0 / (pow(6.0 * ddn, 1.0 / q) + 1e-6);
      }
      if (q < QMAX && qprev == q) {
        const double r = pow(h / hprev, q + 1);
        for (int i = 0; i < NV; ++i) tmp[i] = acor[i] - r * acorp[i];
        const double dup = UPC[q] * wrms(tmp, ewt, NV);
        eta_p = 1.0 / (pow(10.0 * dup, 1.0 / (q + 2)) + 1e-6);
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
    for (int i = 0; i < NV; ++i) acorp[i] = acor[i];
    qprev = q;
    hprev = h;
    if (newq == q + 1) {
      for (int i = 0; i < NV; ++i) z[q + 1][i] = L[q][q] * acor[i] / (q + 1);
      q = q + 1;
      qprev = 0;
    } else if (newq == q - 1) {
      q = q - 1;
      qprev = 0;
    }
    if (eta != 1.0 || qprev == 0)
      qwait = q + 1; /* wait q+1 steps after a change of h or q */
    else if (qwait <= 0)
      qwait = 2; /* order kept: look again two steps later */
    if (eta != 1.0) {
      rescale(z, q, NV, eta);
      h *= eta;
    }
  }
done:
  for (int i = 0; i < NV; ++i) u[i] = z[0][i];
  st->q = q;
  st->h = h;
}

/* Substep over a species-major batch: state[v*ld + i] in/out, dt per cell (or dt_scalar when
 * dts is NULL). OpenMP over cells with dynamic scheduling (stiffness is uneven). */
void orc_bdf_batch(const orc_mech *m, const orc_solver_cfg *cfg, double *state, int64_t ncells, int64_t ld,
                   const double *dts, double dt_scalar, double p, int *nst, int *nni, int *status, int nthreads) {
  const int NV = m->ns + 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
  for (int64_t i = 0; i < ncells; ++i) {
    double u[MAXV];
    orc_cell_stats s;
    for (int v = 0; v < NV; ++v) u[v] = state[v * ld + i];
    orc_bdf_cell(m, cfg, u, dts ? dts[i] : dt_scalar, p, &s);
    for (int v = 0; v < NV; ++v) state[v * ld + i] = u[v];
    if (nst) nst[i] = s.nst;
    if (nni) nni[i] = s.nni;
    if (status) status[i] = s.status;
  }
}
