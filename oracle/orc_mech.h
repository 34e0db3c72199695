/* Flat mechanism tables shared by the oracle's C files -- TEST INFRASTRUCTURE ONLY. */
#ifndef ORC_MECH_H
#define ORC_MECH_H
typedef struct {
  int ns, nslot, nm, nfo;
  double rgas;         /* PRODRATES RGAS and GETLINDRATECOEFF R: literal 8314.34 */
  double troe[7];      /* 0.75, 1.27, 0.4, 0.67, 0.14, 1.0D-60, 1.0 as the literal kinds give */
  const int *tb_ptr, *tb_sp;
  const double *tb_coef;
  const int *k_flags;  /* bit0 falloff, bit1 has n*LT, bit2 has E/RT */
  const double *kA, *kn, *kE;
  const int *k_fo;     /* falloff index of a slot, or -1 */
  const int *f0_flags, *fi_flags;
  const double *f0A, *f0n, *f0E, *fiA, *fin, *fiE;
  const int *fc_ptr, *fc_form; /* form 0: a*exp(-(T/x)), 1: a*exp(-(x/T)) */
  const double *fc_a, *fc_x;
  const int *fo_M;
  const int *w_ptr, *w_sp, *w_M;
  const int *cd_ptr, *cd_sign, *cd_slot;
  const double *cd_coef;
  double tmid;
  const double *th_hi, *th_lo; /* per species 12: c0, a1..a5, a6, b1..b5 */
  const double *wmol;
  const double *nu;  /* ns x nslot, net stoichiometric coefficients (solver Jacobian) */
  const double *eff; /* nm x ns, dense third-body efficiencies (solver Jacobian) */
} orc_mech;
#endif
