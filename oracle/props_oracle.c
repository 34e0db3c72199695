/* CPU FP64 oracle for the mixture properties around the substep -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load this file's library, and
 * only as the checker or the timed CPU baseline; the product never links it.
 *
 * A table-driven restatement, in the reference's statement and operator order, of
 *   - finitechem_W            combustion/finitechem.f90:65-74   (Y clipped to [0,1])
 *   - finitechem_density      finitechem.f90:324-345            (RHO = P W_mix / (R_cst T))
 *   - finitechem_omegamu      finitechem.f90:467-487            (rational collision-integral fit)
 *   - finitechem_viscosity    finitechem.f90:351-406            (Wilke's rule, phi by pow calls)
 *   - finitechem_diffusivity  finitechem.f90:412-461 + finitechem_Cp :79-88
 *                                                               (COMPTHERMODATA inside the species
 *                                                                loop, as :428-432 calls it)
 * R_cst = 8314.34, Tmin = 50, Tmax = 5000 are double parameters (finitechem.f90:7-8, :15). The
 * per-species fits mucoeff / kOverEps (GETMUCOEFF / GETKOVEREPS) and the molar masses come in
 * with the reference's literal kinds from oracle/oracle.py.
 */
#include <math.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "orc_mech.h"

void orc_thermo(const orc_mech *m, double T, double *h, double *cp);

static double omegamu(double temp) {
  const double m1 = 3.3530622607, m2 = 2.53272006, m3 = 2.9024238575, m4 = 0.11186138893, m5 = 0.8662326188;
  const double m6 = 1.3913958626, m7 = 3.158490576, m8 = 0.18973411754, m9 = 0.00018682962894;
  double num = m1 + temp * (m2 + temp * (m3 + temp * m4));
  double den = m5 + temp * (m6 + temp * (m7 + temp * (m8 + temp * m9)));
  return num / den;
}

static double wmix_of(const orc_mech *m, const double *sc) {
  double a = 0.0, b = 0.0;
  for (int k = 0; k < m->ns; ++k) a = a + fmin(fmax(sc[k], 0.0), 1.0);
  for (int k = 0; k < m->ns; ++k) b = b + fmin(fmax(sc[k], 0.0), 1.0) / m->wmol[k];
  return a / b;
}

/* Species-major batch: Y_k of cell c at y[k*ld + c], T at Tin[c]. Each output is nullable:
 * wmix[c], rho[c], visc[c], diff[k*ld + c] = lambda/Cp_mix/lewis[k] (k < ns) and
 * diff[ns*ld + c] = lambda/Cp_mix. lewis nullable (= 1). OpenMP over cells. */
void orc_props_batch(const orc_mech *m, const double *mucoeff, const double *koveps, const double *lewis,
                     const double *y, const double *Tin, int64_t ncells, int64_t ld, double P_thermo, double *wmix,
                     double *rho, double *visc, double *diff, int nthreads) {
  const double R_cst = 8314.34, Tmin = 50.0, Tmax = 5000.0;
  const int ns = m->ns;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t c = 0; c < ncells; ++c) {
    double sc[64], eta[64], cond[64], h_sp[64], Cp_sp[64], phi[64][64];
    for (int k = 0; k < ns; ++k) sc[k] = y[k * ld + c];
    const double T = Tin[c];
    const double W_mix = wmix_of(m, sc);
    if (wmix) wmix[c] = W_mix;
    if (rho) rho[c] = P_thermo * W_mix / (R_cst * T);
    double temp = fmin(fmax(T, Tmin), Tmax);
    if (visc) {
      for (int n = 0; n < ns; ++n) eta[n] = mucoeff[n] * sqrt(temp) / omegamu(temp * koveps[n]);
      for (int k = 0; k < ns; ++k)
        for (int j = 0; j < ns; ++j) {
          phi[k][j] = (1.0 / sqrt(8.0)) * pow(1.0 + (m->wmol[k] / m->wmol[j]), -0.5);
          double temp1 = pow(eta[k] / eta[j], 0.5) * pow(m->wmol[j] / m->wmol[k], 0.25);
          phi[k][j] = phi[k][j] * ((1.0 + temp1) * (1.0 + temp1));
        }
      double sum_2 = 0.0;
      for (int k = 0; k < ns; ++k) {
        double sum_1 = 0.0;
        for (int j = 0; j < ns; ++j)
          if (j != k) sum_1 = sum_1 + (sc[j] * W_mix * phi[k][j] / m->wmol[j]);
        sum_1 = sum_1 + sc[k] * W_mix / m->wmol[k];
        if (sc[k] > 0.0) sum_2 = sum_2 + (sc[k] * W_mix * eta[k] / (m->wmol[k] * sum_1));
      }
      visc[c] = sum_2;
    }
    if (diff) {
      for (int n = 0; n < ns; ++n) {
        eta[n] = mucoeff[n] * sqrt(temp) / omegamu(temp * koveps[n]);
        orc_thermo(m, temp, h_sp, Cp_sp);
        cond[n] = eta[n] * (Cp_sp[n] + 1.25 * R_cst / m->wmol[n]);
      }
      double sum_1 = 0.0, sum_2 = 0.0;
      for (int n = 0; n < ns; ++n) {
        sum_1 = sum_1 + (sc[n] * W_mix / (cond[n] * m->wmol[n]));
        sum_2 = sum_2 + (sc[n] * cond[n] * W_mix / m->wmol[n]);
      }
      double lambda = 0.5 * (sum_2 + (1.0 / sum_1));
      orc_thermo(m, temp, h_sp, Cp_sp);
      double Cp_mix = 0.0;
      for (int n = 0; n < ns; ++n) Cp_mix = Cp_mix + sc[n] * Cp_sp[n];
      for (int n = 0; n < ns; ++n) diff[n * ld + c] = (lambda / Cp_mix) / (lewis ? lewis[n] : 1.0);
      diff[ns * ld + c] = lambda / Cp_mix;
    }
  }
}
