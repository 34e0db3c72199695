/* CPU FP64 oracle for the finite-rate chemistry substep -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load this file's library,
 * and only as the checker or the timed CPU baseline; the product never links it.
 *
 * A table-driven restatement of the reference's per-cell arithmetic, evaluated in the
 * reference's statement and operator order so that it reproduces the reference bit for bit
 * when both use the same libm (compile with -ffp-contract=off):
 *   - PRODRATES            combustion/grimech30F.f90:4-2580 (H2: HYDROGENF.f90:4-277,
 *                          DME: DME39F.f90:4-1943): LT/RT (:29-30), third-body sums (:33-606),
 *                          rate constants (:608-1604), rates (:1605-2028), CDOT (:2029-2579)
 *   - GETLINDRATECOEFF     grimech30F.f90:2583-2619 (Troe branch, ITROE = 1)
 *   - COMPTHERMODATA       grimech30F.f90:2925-3516 (two NASA ranges, T > 1000 strict)
 *   - finitechem_compute_rhs + finitechem_Cp   combustion/finitechem.f90:93-175, :79-88
 *     (low-Mach constant-pressure branch, :160-173)
 * The tables come from the mechanism JSON; oracle/oracle.py turns literals into doubles
 * with the reference's literal kinds and passes flat arrays in an orc_mech.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "orc_mech.h"

static double arrh(int flags, double A, double n, double E, double LT, double RT) {
  if (!(flags & 6)) return A;
  double arg;
  if ((flags & 2) && (flags & 4)) {
    double x = n * LT;
    double y = E / RT;
    arg = x + y;
  } else if (flags & 2) {
    arg = n * LT;
  } else {
    arg = E / RT;
  }
  return A * exp(arg);
}

/* GETLINDRATECOEFF, Troe branch; k0 is overwritten like the Fortran dummy argument. */
static double lind(const orc_mech *m, double T, double P, double *k0, double kinf, double fc, double concin) {
  const double *c = m->troe;
  double conc;
  if (concin > 0.0)
    conc = concin;
  else
    conc = P / (m->rgas * T);
  double ntmp = c[0] - c[1] * log10(fc);
  double cc = -c[2] - c[3] * log10(fc);
  double dc = c[4];
  *k0 = *k0 * conc / fmax(kinf, c[5]);
  double lg = log10(*k0);
  double f = (lg + cc) / (ntmp - dc * (lg + cc));
  f = pow(fc, c[6] / (f * f + c[6]));
  return kinf * f * *k0 / (c[6] + *k0);
}

void orc_thermo(const orc_mech *m, double T, double *h, double *cp) {
  const double *tab = (T > m->tmid) ? m->th_hi : m->th_lo;
  for (int k = 0; k < m->ns; ++k) {
    const double *t = tab + 12 * k;
    h[k] = t[0] * (T * (t[1] + T * (t[2] + T * (t[3] + T * (t[4] + T * (t[5]))))) + t[6]);
    cp[k] = t[0] * (t[7] + T * (t[8] + T * (t[9] + T * (t[10] + T * (t[11])))));
  }
}

/* PRODRATES(CDOT, W, K, C, M, TEMP, PRESSURE); K, W, M are scratch of nslot/nslot/nm. */
void orc_prodrates(const orc_mech *m, double *cdot, double *W, double *K, const double *C, double *M,
                   double T, double P) {
  double LT = log(T);
  double RT = m->rgas * T;
  for (int j = 0; j < m->nm; ++j) {
    int b = m->tb_ptr[j], e = m->tb_ptr[j + 1];
    double acc = m->tb_coef[b] * C[m->tb_sp[b]];
    for (int i = b + 1; i < e; ++i) acc = acc + m->tb_coef[i] * C[m->tb_sp[i]];
    M[j] = acc;
  }
  for (int r = 0; r < m->nslot; ++r) {
    if (m->k_flags[r] & 1) {
      int f = m->k_fo[r];
      double k0 = arrh(m->f0_flags[f], m->f0A[f], m->f0n[f], m->f0E[f], LT, RT);
      double ki = arrh(m->fi_flags[f], m->fiA[f], m->fin[f], m->fiE[f], LT, RT);
      int b = m->fc_ptr[f], e = m->fc_ptr[f + 1];
      double fc = 0.0;
      for (int i = b; i < e; ++i) {
        double t = m->fc_form[i] == 0 ? m->fc_a[i] * exp(-(T / m->fc_x[i])) : m->fc_a[i] * exp(-(m->fc_x[i] / T));
        fc = (i == b) ? t : fc + t;
      }
      K[r] = lind(m, T, P, &k0, ki, fc, M[m->fo_M[f]]);
    } else {
      K[r] = arrh(m->k_flags[r], m->kA[r], m->kn[r], m->kE[r], LT, RT);
    }
  }
  for (int r = 0; r < m->nslot; ++r) {
    double w = K[r];
    for (int i = m->w_ptr[r]; i < m->w_ptr[r + 1]; ++i) w = w * C[m->w_sp[i]];
    if (m->w_M[r] >= 0) w = w * M[m->w_M[r]];
    W[r] = w;
  }
  for (int k = 0; k < m->ns; ++k) {
    int b = m->cd_ptr[k], e = m->cd_ptr[k + 1];
    if (b == e) {
      cdot[k] = 0.0;
      continue;
    }
    double t0 = m->cd_coef[b] * W[m->cd_slot[b]];
    double acc = m->cd_sign[b] < 0 ? -t0 : t0;
    for (int i = b + 1; i < e; ++i) {
      double t = m->cd_coef[i] * W[m->cd_slot[i]];
      acc = m->cd_sign[i] < 0 ? acc - t : acc + t;
    }
    cdot[k] = acc;
  }
}

#define ORC_MAXS 64
#define ORC_MAXR 1024

/* finitechem_compute_rhs (low-Mach branch): sol = (rho*Y_1..N, rho*T) -> rhs. */
void orc_rhs(const orc_mech *m, const double *sol, double p, double *rhs) {
  int N = m->ns;
  double h[ORC_MAXS], cp[ORC_MAXS], Y[ORC_MAXS], conc[ORC_MAXS], cd[ORC_MAXS], M[ORC_MAXS];
  double K[ORC_MAXR], W[ORC_MAXR];
  double rho = 0.0;
  for (int k = 0; k < N; ++k) rho = rho + sol[k];
  for (int k = 0; k < N; ++k) Y[k] = sol[k] / rho;
  double T = sol[N] / rho;
  orc_thermo(m, T, h, cp);
  double cpmix = 0.0;
  for (int k = 0; k < N; ++k) cpmix = cpmix + Y[k] * cp[k];
  for (int k = 0; k < N; ++k) conc[k] = sol[k] / m->wmol[k];
  orc_prodrates(m, cd, W, K, conc, M, sol[N] / rho, p);
  for (int k = 0; k < N; ++k) rhs[k] = cd[k] * m->wmol[k];
  double tmp = 0.0;
  for (int k = 0; k < N; ++k) tmp = tmp - h[k] * rhs[k];
  rhs[N] = tmp / cpmix;
}

/* rhs over a species-major batch: sol[v*ld + i], v = 0..N, i = 0..ncells-1. */
void orc_rhs_batch(const orc_mech *m, const double *sol, double p, double *rhs, int64_t ncells, int64_t ld,
                   int nthreads) {
  int N = m->ns;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < ncells; ++i) {
    double s[ORC_MAXS], r[ORC_MAXS];
    for (int v = 0; v <= N; ++v) s[v] = sol[v * ld + i];
    orc_rhs(m, s, p, r);
    for (int v = 0; v <= N; ++v) rhs[v * ld + i] = r[v];
  }
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Gross (cancellation-free) magnitude of every rhs entry, the denominator of the normwise
 * parity test: gross_k = W_k * sum over the CDOT terms of |coef * W_r|, and
 * gross_T = sum_k |h_k| gross_k / cp_mix. */
void orc_rhs_gross(const orc_mech *m, const double *sol, double p, double *gross) {
  int N = m->ns;
  double h[ORC_MAXS], cp[ORC_MAXS], conc[ORC_MAXS], cd[ORC_MAXS], M[ORC_MAXS];
  double K[ORC_MAXR], W[ORC_MAXR];
  double rho = 0.0;
  for (int k = 0; k < N; ++k) rho = rho + sol[k];
  double T = sol[N] / rho;
  orc_thermo(m, T, h, cp);
  double cpmix = 0.0;
  for (int k = 0; k < N; ++k) cpmix = cpmix + (sol[k] / rho) * cp[k];
  for (int k = 0; k < N; ++k) conc[k] = sol[k] / m->wmol[k];
  orc_prodrates(m, cd, W, K, conc, M, T, p);
  double gt = 0.0;
  for (int k = 0; k < N; ++k) {
    double g = 0.0;
    for (int i = m->cd_ptr[k]; i < m->cd_ptr[k + 1]; ++i) g += fabs(m->cd_coef[i] * W[m->cd_slot[i]]);
    gross[k] = g * m->wmol[k];
    gt += fabs(h[k]) * gross[k];
  }
  gross[N] = gt / cpmix;
}

void orc_rhs_gross_batch(const orc_mech *m, const double *sol, double p, double *gross, int64_t ncells, int64_t ld,
                         int nthreads) {
  int N = m->ns;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < ncells; ++i) {
    double s[ORC_MAXS], r[ORC_MAXS];
    for (int v = 0; v <= N; ++v) s[v] = sol[v * ld + i];
    orc_rhs_gross(m, s, p, r);
    for (int v = 0; v <= N; ++v) gross[v * ld + i] = r[v];
  }
}

/* Rates W_r of every slot for a species-major batch (slot-major output rates[r*ld + i]). */
void orc_rates_batch(const orc_mech *m, const double *sol, double p, double *rates, int64_t ncells, int64_t ld,
                     int64_t ldr, int nthreads) {
  int N = m->ns;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t i = 0; i < ncells; ++i) {
    double conc[ORC_MAXS], cd[ORC_MAXS], M[ORC_MAXS], K[ORC_MAXR], W[ORC_MAXR];
    double rho = 0.0;
    for (int k = 0; k < N; ++k) rho = rho + sol[k * ld + i];
    for (int k = 0; k < N; ++k) conc[k] = sol[k * ld + i] / m->wmol[k];
    orc_prodrates(m, cd, W, K, conc, M, sol[N * ld + i] / rho, p);
    for (int r = 0; r < m->nslot; ++r) rates[r * ldr + i] = W[r];
  }
}
