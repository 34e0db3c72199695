"""CUDA code generator: mechanism table -> straight-line sm_100a device code.

The reference's mechanism files are straight-line generated Fortran (``PRODRATES``,
combustion/grimech30F.f90:4-2580). The GPU path keeps that shape -- one cell per thread,
every rate constant, rate and production rate in registers, every coefficient an immediate --
but generates it from the mechanism table and restructures the arithmetic for the GPU:

* ``K = exp(lnA + n*LT + E*invRT)``: ``ln A`` folded into the exponent (one FMA pair per slot,
  no separate multiply), ``1/(R T)`` formed once per cell instead of one division per slot;
* Troe falloff (GETLINDRATECOEFF, grimech30F.f90:2583-2619) evaluated from the logarithms of
  k0 and kinf directly -- ``log10(Pr) = (ln k0 + ln[M] - ln max(kinf,1e-60))/ln 10`` -- so the
  k0/kinf exponentials and the ``log10`` of the reference collapse into one ``exp`` for Pr; the
  centring factor F_cent and its logarithm are computed once per distinct F_cent expression
  (a forward/reverse pair shares one);
* production rates accumulated by scatter right after each rate ``W_r`` is formed (net
  stoichiometric coefficient per species and slot), so W never has to be stored;
* thermodynamics (COMPTHERMODATA, grimech30F.f90:2925-3516) evaluated after the rates for the
  enthalpy term of the temperature equation (finitechem.f90:160-173).

Two precision modes are emitted per mechanism:

``rhs_fp64`` -- everything in FP64; agrees with the reference arithmetic to ~1e-14 relative.

``rhs_mixed`` -- every rate is formed in base-2 log space and exponentiated with the FP32
``ex2.approx`` unit: forward (and irreversible) slots assemble their exponent in FP32; the
fitted reverse slots -- whose ``ln A_b - E_b/RT`` carries the large cancellations the
equilibrium constant was folded into -- assemble it in FP64 and round only the final exponent.
Third-body sums, production-rate accumulation and thermodynamics stay FP64.

Both take ``LM`` (literal mode) as a template argument: 0 = reference literal kinds, 1 = all
literals double. Generated files go to ``tiger_nga_b200/_build/gen``; they are rebuilt from the
committed tables by :mod:`tiger_nga_b200.build`.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

from .mechanism import Mechanism

LOG2E = 1.0 / math.log(2.0)
INV_LN10 = 1.0 / math.log(10.0)
LOG10_2 = math.log10(2.0)


def _d(x: float) -> str:
    if x == 0.0:
        return "0.0"
    return float(x).hex()


def _f(x: float) -> str:
    v = float(np.float32(x))
    if v == 0.0:
        return "0.0f"
    return v.hex() + "f"


def _lm(a: float, b: float, fmt=_d) -> str:
    """Literal-mode select between the reference-kind value a and the all-double value b."""
    sa, sb = fmt(a), fmt(b)
    return sa if sa == sb else f"TNG_LM({sa}, {sb})"


class _Gen:
    def __init__(self, name: str):
        self.name = name
        self.m32 = Mechanism(name, "f32")
        self.m64 = Mechanism(name, "f64")
        m = self.m32
        self.ns, self.nslot, self.nm = m.ns, m.nslot, m.nm
        # first slot that needs each third-body set (as W factor or as falloff [M])
        self.fc_keys32: dict[tuple, int] = {}

    # ---------------------------------------------------------------- helpers
    def arr_terms(self, a32, a64, log2: bool):
        """(lnA, n, E) constant strings; log2=True scales to base-2 units."""
        s = LOG2E if log2 else 1.0
        lnA = _lm(math.log(a32.A) * s, math.log(a64.A) * s)
        n = _lm(a32.n, a64.n) if a32.n is not None else None
        E = _lm(a32.E * s, a64.E * s) if a32.E is not None else None
        return lnA, n, E

    def fc_code(self, idx: int, fc32, fc64, out: list[str], prec: str):
        """Emit F_cent for one distinct expression; returns the names of log10(fc), log2(fc)."""
        terms = []
        for (a, form, x), (a6, _, x6) in zip(fc32, fc64):
            # exact shortcuts: exp(-T/1e30) == 1.0 and exp(-T/1e-30) == 0.0 in double for any T in range
            if form == 0 and x <= 1e-20:
                continue
            if form == 1 and x >= 1e20:
                continue
            if (form == 0 and x >= 1e20) or (form == 1 and x == 0.0):
                terms.append(_lm(a, a6))
                continue
            if form == 0:
                terms.append(f"{_lm(a, a6)} * exp(-T * {_lm(1.0 / x, 1.0 / x6)})")
            else:
                terms.append(f"{_lm(a, a6)} * exp(-{_lm(x, x6)} * invT)")
        if not terms:
            raise ValueError("F_cent is identically zero")
        out.append(f"  const double fc{idx} = {' + '.join(terms)};")
        out.append(f"  const double lfc{idx} = log(fc{idx});")
        out.append(f"  const double l10fc{idx} = lfc{idx} * {_d(INV_LN10)};")
        out.append(f"  const double ntmp{idx} = {_lm(self.m32.troe['c_n0'], self.m64.troe['c_n0'])} - "
                   f"{_lm(self.m32.troe['c_n1'], self.m64.troe['c_n1'])} * l10fc{idx};")
        out.append(f"  const double cc{idx} = -{_lm(self.m32.troe['c_c0'], self.m64.troe['c_c0'])} - "
                   f"{_lm(self.m32.troe['c_c1'], self.m64.troe['c_c1'])} * l10fc{idx};")
        if prec == "mixed":
            out.append(f"  const float l2fcf{idx} = (float)(lfc{idx} * {_d(LOG2E)});")
            out.append(f"  const float ntmpf{idx} = (float)ntmp{idx};")
            out.append(f"  const float ccf{idx} = (float)cc{idx};")

    # ---------------------------------------------------------------- one rhs function
    def rhs(self, prec: str, dump: bool = False) -> str:
        m32, m64 = self.m32, self.m64
        ns = self.ns
        o: list[str] = []
        fn = f"rhs_{prec}"
        o.append(f"template <int LM, bool DUMP, int SYNC>")
        o.append(f"__device__ static __forceinline__ void {fn}(const double* __restrict__ s, double p, double* __restrict__ r,"
                 f" double* __restrict__ dump, long long dld) {{")
        o.append("  (void)dump; (void)dld;")
        # rho and T
        o.append("  double rho = s[0];")
        for k in range(1, ns):
            o.append(f"  rho = rho + s[{k}];")
        o.append("  const double irho = 1.0 / rho;")
        o.append(f"  // T by division, as the reference forms it: the strict T > 1000 range switch of the")
        o.append(f"  // NASA polynomials must see the same value")
        o.append(f"  const double T = s[{ns}] / rho;")
        o.append("  const double LT = log(T);")
        o.append(f"  const double invRT = 1.0 / ({_lm(m32.rgas, m64.rgas)} * T);")
        o.append(f"  const double invT = {_lm(m32.rgas, m64.rgas)} * invRT;")
        for k in range(ns):
            o.append(f"  const double c{k} = s[{k}] * {_lm(1.0 / m32.wmol[k], 1.0 / m64.wmol[k])};")
            o.append(f"  double cd{k} = 0.0;")
        if prec == "mixed":
            o.append("  const float LT2f = (float)(LT * %s);" % _d(LOG2E))
            o.append("  const double LT2 = LT * %s;" % _d(LOG2E))
            o.append("  const float invRTf = (float)invRT;")
            for k in range(ns):
                o.append(f"  const float lc{k} = tng_lg2f(fabsf((float)c{k}));")
                o.append(f"  const float sg{k} = c{k} < 0.0 ? -1.0f : 1.0f;")
        have_m: set[int] = set()
        have_lc: set[int] = set()
        have_fc: dict[tuple, int] = {}
        lnprt_done = False

        def need_m(j):
            if j in have_m:
                return
            terms = m32.third_body[j]
            terms64 = m64.third_body[j]
            parts = []
            for (s_, c), (_, c6) in zip(terms, terms64):
                parts.append(f"c{s_}" if c == 1.0 and c6 == 1.0 else f"{_lm(c, c6)} * c{s_}")
            o.append(f"  const double m{j} = {' + '.join(parts)};")
            if prec == "mixed":
                o.append(f"  const float lm{j} = tng_lg2f(fabsf((float)m{j}));")
                o.append(f"  const float sm{j} = m{j} < 0.0 ? -1.0f : 1.0f;")
            have_m.add(j)

        for s32, s64 in zip(m32.slots, m64.slots):
            r = s32.index
            if r > 0 and r % 48 == 0:
                o.append("  if constexpr (SYNC != 0) __syncthreads();  // keep the block's warps on the same code lines")
            o.append(f"  // slot {r}: {s32.name}")
            reverse = s32.reverse
            if s32.kind == "falloff":
                need_m(s32.M_fall)
                if s32.M >= 0:
                    need_m(s32.M)
                if not lnprt_done:
                    o.append("  const double lnprt = log(p * invRT);")
                    lnprt_done = True
                j = s32.M_fall
                if j not in have_lc:
                    o.append(f"  const double lcm{j} = m{j} > 0.0 ? log(m{j}) : lnprt;")
                    have_lc.add(j)
                key = s32.fc_key
                lind = key == ((1.0, 1, 0.0),)  # F_cent == 1: plain Lindemann
                if not lind and key not in have_fc:
                    have_fc[key] = len(have_fc)
                    self.fc_code(have_fc[key], s32.fc, s64.fc, o, prec)
                lnA0, n0, E0 = self.arr_terms(s32.k0, s64.k0, False)
                lnAi, ni, Ei = self.arr_terms(s32.kinf, s64.kinf, False)

                def expo(lnA, n, E):
                    e = lnA
                    if E is not None:
                        e = f"fma({E}, invRT, {e})"
                    if n is not None:
                        e = f"fma({n}, LT, {e})"
                    return e

                kmin = math.log(m32.troe["kmin"])
                o.append(f"  {{ const double lk0 = {expo(lnA0, n0, E0)};")
                o.append(f"    const double lki = {expo(lnAi, ni, Ei)};")
                o.append(f"    const double lpr = lk0 + lcm{j} - fmax(lki, {_d(kmin)});")
                if prec == "fp64":
                    o.append("    const double pr = exp(lpr);")
                    if lind:
                        o.append("    double w = exp(lki) * pr / (1.0 + pr);")
                    else:
                        u = have_fc[key]
                        o.append(f"    const double lg = lpr * {_d(INV_LN10)} + cc{u};")
                        o.append(f"    const double f = lg / (ntmp{u} - {_lm(m32.troe['c_d'], m64.troe['c_d'])} * lg);")
                        o.append(f"    double w = exp(lki + lfc{u} / (f * f + 1.0)) * pr / (1.0 + pr);")
                    for c in s32.C:
                        o.append(f"    w = w * c{c};")
                    if s32.M >= 0:
                        need_m(s32.M)
                        o.append(f"    w = w * m{s32.M};")
                else:
                    # FP64 exponents of k0/kinf, Troe blending in FP32 base-2 logs
                    o.append("    const float lpr2 = (float)(lpr * %s);" % _d(LOG2E))
                    o.append("    const float lki2 = (float)(lki * %s);" % _d(LOG2E))
                    if lind:
                        o.append("    const float lk2 = lki2 + lpr2 - tng_softplus2f(lpr2);")
                    else:
                        u = have_fc[key]
                        o.append(f"    const float lg = lpr2 * {_f(LOG10_2)} + ccf{u};")
                        o.append(f"    const float f = __fdividef(lg, ntmpf{u} - {_f(m32.troe['c_d'])} * lg);")
                        o.append(f"    const float lk2 = lki2 + __fdividef(l2fcf{u}, f * f + 1.0f) + lpr2 - tng_softplus2f(lpr2);")
                    if s32.M >= 0:
                        need_m(s32.M)
                    tail = "".join(f" + lc{c}" for c in s32.C) + (f" + lm{s32.M}" if s32.M >= 0 else "")
                    sg = "".join(f" * sg{c}" for c in s32.C) + (f" * sm{s32.M}" if s32.M >= 0 else "")
                    o.append(f"    const double w = (double)(tng_ex2f(lk2{tail}){sg});")
                if dump:
                    o.append(f"    if (DUMP && dump) dump[{r}LL * dld] = w;  // null for the lanes past the last cell")
                self.scatter(r, o, "    ")
                o.append("  }")
                continue

            a32, a64 = s32.arr, s64.arr
            if s32.M >= 0:
                need_m(s32.M)
            if prec == "fp64":
                if a32.n is None and a32.E is None:
                    o.append(f"  {{ double w = {_lm(a32.A, a64.A)};")
                else:
                    lnA, n, E = self.arr_terms(a32, a64, False)
                    e = lnA
                    if E is not None:
                        e = f"fma({E}, invRT, {e})"
                    if n is not None:
                        e = f"fma({n}, LT, {e})"
                    o.append(f"  {{ double w = exp({e});")
                for c in s32.C:
                    o.append(f"    w = w * c{c};")
                if s32.M >= 0:
                    o.append(f"    w = w * m{s32.M};")
            else:
                lnA, n, E = self.arr_terms(a32, a64, True)
                if reverse:
                    e = lnA
                    if E is not None:
                        e = f"fma({E}, invRT, {e})"
                    if n is not None:
                        e = f"fma({n}, LT2, {e})"
                    head = f"(float)({e})"
                else:
                    lnAf = _lm(math.log(a32.A) * LOG2E, math.log(a64.A) * LOG2E, _f)
                    e = lnAf
                    if E is not None:
                        e = f"fmaf({_lm(a32.E * LOG2E, a64.E * LOG2E, _f)}, invRTf, {e})"
                    if n is not None:
                        e = f"fmaf({_lm(a32.n, a64.n, _f)}, LT2f, {e})"
                    head = e
                tail = "".join(f" + lc{c}" for c in s32.C) + (f" + lm{s32.M}" if s32.M >= 0 else "")
                sg = "".join(f" * sg{c}" for c in s32.C) + (f" * sm{s32.M}" if s32.M >= 0 else "")
                o.append(f"  {{ const double w = (double)(tng_ex2f({head}{tail}){sg});")
            if dump:
                o.append(f"    if (DUMP && dump) dump[{r}LL * dld] = w;  // null for the lanes past the last cell")
            self.scatter(r, o, "    ")
            o.append("  }")

        # epilogue: production rates -> mass rates, temperature equation
        o.append("  double cpm = 0.0, tmp = 0.0;")
        o.append(f"  if (T > {_lm(m32.tmid, m64.tmid)}) {{")
        self.thermo_block(m32.th_hi, m64.th_hi, o)
        o.append("  } else {")
        self.thermo_block(m32.th_lo, m64.th_lo, o)
        o.append("  }")
        o.append(f"  r[{ns}] = tmp / cpm;")
        o.append("}")
        return "\n".join(o)

    def scatter(self, r: int, o: list[str], ind: str):
        col = self.m32.nu[:, r]
        col64 = self.m64.nu[:, r]
        for k in range(self.ns):
            v, v6 = col[k], col64[k]
            if v == 0.0 and v6 == 0.0:
                continue
            if v == 1.0 and v6 == 1.0:
                o.append(f"{ind}cd{k} += w;")
            elif v == -1.0 and v6 == -1.0:
                o.append(f"{ind}cd{k} -= w;")
            else:
                o.append(f"{ind}cd{k} = fma({_lm(v, v6)}, w, cd{k});")

    def thermo_block(self, t32, t64, o):
        m32, m64 = self.m32, self.m64
        for k in range(self.ns):
            a, b = t32[k], t64[k]
            L = lambda i: _lm(a[i], b[i])  # noqa: E731
            o.append(f"    {{ const double y = c{k} * ({_lm(m32.wmol[k], m64.wmol[k])} * irho);")
            o.append(f"      const double cpk = {L(0)} * ({L(7)} + T * ({L(8)} + T * ({L(9)} + T * ({L(10)} + T * {L(11)}))));")
            o.append(f"      const double hk = {L(0)} * (T * ({L(1)} + T * ({L(2)} + T * ({L(3)} + T * ({L(4)} + T * {L(5)})))) + {L(6)});")
            o.append(f"      const double rk = cd{k} * {_lm(m32.wmol[k], m64.wmol[k])};")
            o.append(f"      r[{k}] = rk;")
            o.append(f"      cpm = fma(y, cpk, cpm);")
            o.append(f"      tmp = fma(-hk, rk, tmp); }}")

    # ---------------------------------------------------------------- mixture properties
    def props(self) -> str:
        """Per-cell mixture properties around the substep (finitechem.f90:65-74, :324-487).

        ``mix_w``: W_mix of the clipped mass fractions (finitechem_W). ``transport``: the species
        viscosities eta_k = mucoeff_k sqrt(T) / Omega(T kOverEps_k) (finitechem_omegamu's rational
        fit), then
        * the conductivity sums, Cp_mix and lambda/Cp_mix of finitechem_diffusivity;
        * Wilke's mixture viscosity of finitechem_viscosity. Its pair factor
          phi_kj = A_kj (1 + sqrt(eta_k/eta_j) (W_j/W_k)^1/4)^2, A_kj = (1 + W_k/W_j)^-1/2 / sqrt(8),
          is rewritten with q = W^1/4 as A_kj (1 + sig_k rho_j)^2, rho = q/sqrt(eta), sig = 1/rho,
          so that sum_j x_j phi_kj = A.u + 2 sig_k A.(u rho) + sig_k^2 A.(u rho^2):
          three dot products of per-cell vectors with ONE constant matrix A (zero diagonal: the
          reference's j /= k), three FMAs per pair instead of the reference's three pow calls.
          W_mix cancels between sum_1 and sum_2 and is left out, and with rho_k = v_k/u_k,
          rho_k^2 = w_k/u_k row k's term u_k eta_k / sum_1 becomes
          u_k^2 q_k^2 / (w_k (u_k + A.u) + 2 v_k A.(u rho) + u_k A.(u rho^2)): one division. The
          per-cell vectors u, v = u rho, w = v rho live in shared memory (stride B, one slice per
          thread); rows run in tiles of up to 13 (a runtime loop, A read from constant memory at a
          warp-uniform address), so each vector load feeds up to 39 FMAs and the code stays
          small enough for the instruction cache.
        """
        m32, m64 = self.m32, self.m64
        ns = self.ns
        o: list[str] = []
        om = {i + 1: v for i, v in enumerate((3.3530622607, 2.53272006, 2.9024238575, 0.11186138893, 0.8662326188,
                                              1.3913958626, 3.158490576, 0.18973411754, 0.00018682962894))}
        o.append("  template <int LM>")
        o.append("  __device__ static __forceinline__ double mix_w(const double* __restrict__ y, long long ld) {")
        o.append("    double st = 0.0, sw = 0.0;")
        o.append("#pragma unroll 4")
        o.append(f"    for (int k = 0; k < {ns}; ++k) {{")
        o.append("      const double t = fmin(fmax(__ldcs(y + k * ld), 0.0), 1.0);")
        o.append(f"      st = st + t; sw = fma(t, {self.name}_props_records[LM][19 * k + 2], sw);")
        o.append("    }")
        o.append("    return st / sw;")
        o.append("  }")
        # the species loop is a runtime loop over per-species records in constant memory
        # (props_records): unrolled, the scheduler would keep every species' fit live at once
        o.append("  template <int LM, bool VISC, bool DIFF, int B>")
        o.append("  __device__ static __forceinline__ void transport(const double* __restrict__ y, long long ldy, double T,"
                 " double* __restrict__ sv, double* visc, double* lam_cp) {")
        o.append("    const double Tc = fmin(fmax(T, 50.0), 5000.0);  // Tmin, Tmax (finitechem.f90:7-8)")
        o.append("    const double sq = sqrt(Tc);")
        o.append(f"    const int toff = Tc > {_lm(m32.tmid, m64.tmid)} ? 4 : 10;")
        o.append("    double s1 = 0.0, s2 = 0.0, cpm = 0.0, st = 0.0, sw = 0.0;")
        o.append("    // stage the mass fractions in this thread's shared-memory slice first (all loads in")
        o.append("    // flight at once; the species loop below would otherwise wait on each in turn)")
        o.append("    constexpr int SV = VISC ? 3 : 1;")
        o.append("#pragma unroll")
        o.append(f"    for (int k = 0; k < {ns}; ++k) sv[SV * k * B] = __ldcs(y + k * ldy);")
        o.append("#pragma unroll 4  // four species' dependent chains (fit, division, rsqrt) interleaved")
        o.append(f"    for (int k = 0; k < {ns}; ++k) {{")
        o.append(f"      const double* q = {self.name}_props_records[LM] + 19 * k;")
        o.append("      const double yk = sv[SV * k * B];")
        o.append("      const double x = Tc * q[0];")
        o.append(f"      const double num = fma(x, fma(x, fma(x, {_d(om[4])}, {_d(om[3])}), {_d(om[2])}), {_d(om[1])});")
        o.append(f"      const double den = fma(x, fma(x, fma(x, fma(x, {_d(om[9])}, {_d(om[8])}), {_d(om[7])}), "
                 f"{_d(om[6])}), {_d(om[5])});")
        o.append("      const double e = q[1] * sq * den / num;  // mucoeff sqrt(T) / Omega(T kOverEps)")
        o.append("      const double u = yk * q[2];")
        o.append("      if (VISC) {  // u, u rho, u rho^2 with rho = q/sqrt(eta)")
        o.append("        const double r = rsqrt(e) * q[16];")
        o.append("        const double v = u * r;")
        o.append("        sv[3 * k * B] = u; sv[(3 * k + 1) * B] = v; sv[(3 * k + 2) * B] = v * r;")
        o.append("      }")
        o.append("      if (DIFF) {")
        o.append("        const double* a = q + toff;")
        o.append("        const double cp = a[0] * (a[1] + Tc * (a[2] + Tc * (a[3] + Tc * (a[4] + Tc * a[5]))));")
        o.append("        const double c = e * (cp + q[3]);")
        o.append("        s1 = s1 + u / c; s2 = fma(u, c, s2); cpm = fma(yk, cp, cpm);")
        o.append("        const double t = fmin(fmax(yk, 0.0), 1.0); st = st + t; sw = fma(t, q[2], sw);")
        o.append("      }")
        o.append("    }")
        o.append("    if (DIFF) { const double wmix = st / sw; *lam_cp = (0.5 * (wmix * s2 + 1.0 / (wmix * s1))) / cpm; }")
        R, nrow = self.wilke_tile()
        o.append("    if (VISC) {")
        o.append("      double acc = 0.0;")
        o.append("#pragma unroll 1")
        o.append(f"      for (int k0 = 0; k0 < {ns}; k0 += {R}) {{")
        o.append(f"        const double* A = {self.name}_wilke[LM] + k0 * {ns};")
        o.append("        " + " ".join(f"double a{r} = 0.0, b{r} = 0.0, c{r} = 0.0;" for r in range(R)))

        def loads(jj):
            o.append(f"        const double u{jj} = sv[{3 * jj} * B], v{jj} = sv[{3 * jj + 1} * B], "
                     f"w{jj} = sv[{3 * jj + 2} * B];")
            o.append("        const double " + ", ".join(f"m{jj}_{r} = A[{r * ns + jj}]" for r in range(R)) + ";")

        # software-pipelined columns: column j+1's loads are issued before column j's FMAs, and
        # a scheduling fence keeps the compiler from hoisting further ahead (registers)
        loads(0)
        for jj in range(ns):
            if jj + 1 < ns:
                loads(jj + 1)
            o.append("        TNG_SCHED_FENCE();")
            for r in range(R):
                o.append(f"        a{r} = fma(m{jj}_{r}, u{jj}, a{r}); b{r} = fma(m{jj}_{r}, v{jj}, b{r}); "
                         f"c{r} = fma(m{jj}_{r}, w{jj}, c{r});")
        for r in range(R):
            o.append(f"        if (k0 + {r} < {ns}) {{")
            o.append(f"          const int k = k0 + {r};")
            o.append("          const double uk = sv[3 * k * B];")
            o.append("          // u eta / sum_1 with eta = q^2 / rho^2, rho = v/u, rho^2 = w/u (rows with u <= 0 add nothing)")
            o.append("          if (uk > 0.0) {")
            o.append("            const double vk = sv[(3 * k + 1) * B], wk = sv[(3 * k + 2) * B];")
            o.append(f"            acc += uk * uk * {self.name}_props_records[LM][19 * k + 18] / "
                     f"fma(wk, uk + a{r}, fma(2.0 * b{r}, vk, c{r} * uk));")
            o.append("          }")
            o.append("        }")
        o.append("      }")
        o.append("      *visc = acc;")
        o.append("    }")
        o.append("  }")
        return "\n".join(o)

    def wilke_tile(self):
        """Rows per tile of the Wilke sum (at most 13, three accumulators each) and the padded
        row count of the matrix."""
        ntiles = -(-self.ns // 13)
        R = -(-self.ns // ntiles)
        return R, R * ntiles

    def props_records(self) -> str:
        """Per-species records of ``transport``, [literal mode][species x 19]: kOverEps,
        mucoeff, 1/W, 1.25 R_cst/W (finitechem.f90:431), the NASA cp coefficients c0, b1..b5 of
        the high and of the low range, then q = W^1/4, 1/q and q^2 (Wilke's rewritten factor).
        And Wilke's matrix A_kj = (1 + W_k/W_j)^-1/2 / sqrt(8) with a zero diagonal, rows padded to
        a whole number of tiles with zeros, [literal mode][row x N]."""
        rc = 8314.34
        ns = self.ns
        nrow = self.wilke_tile()[1]

        def rec(m, k):
            q = m.wmol[k] ** 0.25
            return ([m.koveps[k], m.mucoeff[k], 1.0 / m.wmol[k], 1.25 * rc / m.wmol[k]]
                    + [m.th_hi[k][i] for i in (0, 7, 8, 9, 10, 11)] + [m.th_lo[k][i] for i in (0, 7, 8, 9, 10, 11)]
                    + [q, 1.0 / q, q * q])

        def wilke(m):
            A = np.zeros((nrow, ns))
            for k in range(ns):
                for j in range(ns):
                    if j != k:
                        A[k, j] = (1.0 / math.sqrt(8.0)) * (1.0 + m.wmol[k] / m.wmol[j]) ** -0.5
            return A

        recs = ["{" + ", ".join(_d(v) for k in range(ns) for v in rec(mm, k)) + "}" for mm in (self.m32, self.m64)]
        mats = ["{" + ", ".join(_d(v) for v in wilke(mm).ravel()) + "}" for mm in (self.m32, self.m64)]
        return (f"// per-species records of Mech_{self.name}::transport, [literal mode][species][19]\n"
                f"static __constant__ double {self.name}_props_records[2][{ns * 19}] = {{{', '.join(recs)}}};\n"
                f"// Wilke's matrix of Mech_{self.name}::transport, [literal mode][row][species]\n"
                f"static __constant__ double {self.name}_wilke[2][{nrow * ns}] = {{{', '.join(mats)}}};")

    def header(self) -> str:
        m32, m64 = self.m32, self.m64
        cls = f"Mech_{self.name}"
        out = [f"// Generated from tiger_nga_b200/mechanisms/{self.name}.json by tiger_nga_b200/codegen.py.",
               "// Do not edit: regenerate with tiger_nga_b200.build.",
               "#pragma once",
               '#include "tng_device.cuh"',
               "namespace tng {",
               self.props_records(),
               f"struct {cls} {{",
               f"  static constexpr int NS = {self.ns};",
               f"  static constexpr int NSLOT = {self.nslot};",
               f"  static constexpr int NM = {self.nm};",
               f'  static constexpr const char* NAME = "{self.name}";']
        out.append(self.rhs("fp64", dump=True))
        out.append(self.rhs("mixed", dump=True))
        out.append(self.props())
        out.append("};")
        # host-side info
        names = ", ".join(f'"{s}"' for s in m32.species)
        out.append(f"static const char* const {self.name}_species[{self.ns}] = {{{names}}};")
        out.append(f"static const double {self.name}_wmol[2][{self.ns}] = {{{{{', '.join(_d(x) for x in m32.wmol)}}}, "
                   f"{{{', '.join(_d(x) for x in m64.wmol)}}}}};")
        el = m32.elem
        out.append(f"static const int {self.name}_nelem = {el.shape[0]};")
        out.append(f'static const char* const {self.name}_elements[{el.shape[0]}] = {{{", ".join(chr(34) + e + chr(34) for e in m32.elements)}}};')
        out.append(f"static const double {self.name}_elem[{el.shape[0]}][{self.ns}] = {{"
                   + ", ".join("{" + ", ".join(_d(x) for x in row) + "}" for row in el) + "};")
        out.append("}  // namespace tng")
        return "\n".join(out) + "\n"


def generate(name: str) -> str:
    return _Gen(name).header()


def write_all(out_dir: str, names=("hydrogen", "grimech30", "dme39")) -> list[str]:
    os.makedirs(out_dir, exist_ok=True)
    paths = []
    for n in names:
        for fname, src in ((f"mech_{n}.cuh", generate(n)), (f"solver_{n}.h", solver_header(n))):
            path = os.path.join(out_dir, fname)
            old = open(path).read() if os.path.exists(path) else None
            if old != src:
                with open(path, "w") as fh:
                    fh.write(src)
            paths.append(path)
    return paths



# ---------------------------------------------------------------------------------------------
# Tables of the warp-cooperative implicit solver (csrc/solver.cuh)
# ---------------------------------------------------------------------------------------------
#
# Slots are renumbered into a processing order (falloff, then exponential Arrhenius, then
# constant rate constants) so that the 32 lanes of a round take the same branch; every table
# below is indexed by that position p. "Hot" tables (everything the right-hand side touches) are
# staged into shared memory once per block; "cold" tables (the Jacobian's work lists) are read
# through L1. Stoichiometric coefficients are small integers and are packed into the index words.

NONE7 = 127


def _layout_const(name: str) -> int:
    """A record stride of csrc/solver_layout.h (the one place it is defined)."""
    import re
    src = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "solver_layout.h")).read()
    return int(re.search(rf"\b{name} = (\d+)", src).group(1))


# Odd record strides: the lanes reading one field of consecutive records hit distinct banks.
SLOT_REC, FO_REC, FC_REC, TH_STRIDE = (_layout_const(k) for k in ("kSlotRec", "kFoRec", "kFcRec", "kThStride"))
assert SLOT_REC == 3 and FO_REC == 7 and FC_REC == 7 and TH_STRIDE >= 24


def _lpt(sizes: list[int], nlanes: int = 32) -> list[list[int]]:
    """Longest-processing-time assignment of tasks to lanes (deterministic)."""
    order = sorted(range(len(sizes)), key=lambda t: (-sizes[t], t))
    load = [0] * nlanes
    lanes: list[list[int]] = [[] for _ in range(nlanes)]
    for t in order:
        L = min(range(nlanes), key=lambda x: (load[x], x))
        lanes[L].append(t)
        load[L] += sizes[t]
    return [sorted(x) for x in lanes]


def _nu8(v: float) -> int:
    iv = int(round(v))
    if iv != v or not -127 <= iv <= 127:
        raise ValueError("stoichiometric coefficient is not a small integer")
    return iv & 0xFF


def solver_tables(name: str) -> dict:
    g = _Gen(name)
    m32, m64 = g.m32, g.m64
    ns, nslot, nm = g.ns, g.nslot, g.nm
    nv = ns + 1
    if ns >= NONE7 or nm >= NONE7:
        raise ValueError("too many species or third-body sets for the packed solver tables")

    def kind(s):
        if s.kind == "falloff":
            return 0
        return 2 if (s.arr.n is None and s.arr.E is None) else 1

    order = sorted(range(nslot), key=lambda r: (kind(m32.slots[r]), r))
    pos = {r: p for p, r in enumerate(order)}
    hd = {}  # name -> [list32, list64]
    hi = {}
    ci = {}

    def HD(key, v32, v64):
        hd[key] = [list(map(float, v32)), list(map(float, v64))]

    # slots (processing order)
    sd32, sd64, si = [], [], []
    fos = []
    for r in order:
        s32, s64 = m32.slots[r], m64.slots[r]
        reac = (s32.C + [NONE7] * 3)[:3]
        mw = s32.M if s32.M >= 0 else NONE7
        if s32.kind == "falloff":  # the falloff slots come first and have no plain record
            flags, fo = 1, len(fos)
            fos.append((s32, s64))
        else:
            a, b = s32.arr, s64.arr
            flags = (2 if a.n is not None else 0) | (4 if a.E is not None else 0)
            fo = 0
            if flags == 0:
                flags = 8
                sd32 += [a.A, 0.0, 0.0]
                sd64 += [b.A, 0.0, 0.0]
            else:
                sd32 += [math.log(a.A), a.E or 0.0, a.n or 0.0]
                sd64 += [math.log(b.A), b.E or 0.0, b.n or 0.0]
        si += [flags | (reac[0] << 4) | (reac[1] << 11) | (reac[2] << 18), mw | (fo << 8)]
    HD("slot", sd32, sd64)
    hi["slot"] = si

    fc_ids: dict[tuple, int] = {}
    fcd32, fcd64, fci = [], [], []
    fod32, fod64, foi = [], [], []
    for s32, s64 in fos:
        fl = []
        for a, b in ((s32.k0, s64.k0), (s32.kinf, s64.kinf)):
            fl.append((2 if a.n is not None else 0) | (4 if a.E is not None else 0))
            fod32 += [math.log(a.A), a.E or 0.0, a.n or 0.0]
            fod64 += [math.log(b.A), b.E or 0.0, b.n or 0.0]
        fod32.append(0.0), fod64.append(0.0)  # pad to FO_REC
        key = s32.fc_key
        if key == ((1.0, 1, 0.0),):
            fcid = -1
        else:
            if key not in fc_ids:
                fc_ids[key] = len(fc_ids)
                forms, r32, r64 = [], [], []
                for (a, form, x), (a6, _, x6) in zip(s32.fc, s64.fc):
                    if form == 0 and x <= 1e-20:
                        continue
                    if form == 1 and x >= 1e20:
                        continue
                    if (form == 0 and x >= 1e20) or (form == 1 and x == 0.0):
                        forms.append(2), r32.append((a, 0.0)), r64.append((a6, 0.0))
                    elif form == 0:
                        forms.append(0), r32.append((a, 1.0 / x)), r64.append((a6, 1.0 / x6))
                    else:
                        forms.append(1), r32.append((a, x)), r64.append((a6, x6))
                assert 1 <= len(forms) <= 3
                while len(forms) < 3:
                    forms.append(15), r32.append((0.0, 0.0)), r64.append((0.0, 0.0))
                fci.append(forms[0] | (forms[1] << 4) | (forms[2] << 8))
                fcd32 += [v for t in r32 for v in t] + [0.0]  # pad to FC_REC
                fcd64 += [v for t in r64 for v in t] + [0.0]
            fcid = fc_ids[key]
        foi.append(fl[0] | (fl[1] << 4) | ((fcid + 1) << 8) | (s32.M_fall << 16))
    HD("fo", fod32, fod64)
    hi["fo"] = foi
    HD("fc", fcd32, fcd64)
    hi["fc"] = fci
    nfo, nfc = len(fos), len(fc_ids)

    eff32 = np.zeros((max(nm, 1), ns | 1))  # rows of eff_stride(ns) = ns | 1
    eff64 = np.zeros((max(nm, 1), ns | 1))
    for j, (t32, t64) in enumerate(zip(m32.third_body, m64.third_body)):
        for (s_, c), (_, c6) in zip(t32, t64):
            eff32[j, s_] += c
            eff64[j, s_] += c6
    HD("eff", eff32.reshape(-1), eff64.reshape(-1))
    pad = np.zeros((ns, TH_STRIDE - 24))
    th32 = np.concatenate([m32.th_hi, m32.th_lo, pad], axis=1).reshape(-1)
    th64 = np.concatenate([m64.th_hi, m64.th_lo, pad], axis=1).reshape(-1)
    HD("th", th32, th64)
    HD("wmol", m32.wmol, m64.wmol)
    HD("invw", 1.0 / m32.wmol, 1.0 / m64.wmol)
    sc = []
    for mm in (m32, m64):
        t = mm.troe
        sc.append([mm.rgas, mm.tmid, t["c_n0"], t["c_n1"], t["c_c0"], t["c_c1"], t["c_d"], math.log(t["kmin"]),
                   INV_LN10])
    hd["scal"] = sc

    # production rates: species rows split into chunks, chunks balanced over lanes
    if not np.array_equal(m32.nu, m64.nu):
        raise ValueError("stoichiometry depends on the literal mode")
    nu = m32.nu
    total = int((nu != 0).sum())
    chunk = max(8, -(-total // 32))
    cbeg, cend, cterm, spp = [], [], [], [0]
    for k in range(ns):
        ps = sorted(pos[r] for r in range(nslot) if nu[k, r] != 0.0)
        for b in range(0, len(ps), chunk):
            cbeg.append(len(cterm))
            for p in ps[b:b + chunk]:
                cterm.append((p << 8) | _nu8(nu[k, order[p]]))
            cend.append(len(cterm))
        spp.append(len(cbeg))
    lanes = _lpt([e - b for b, e in zip(cbeg, cend)])
    # interleaved: step s of lane L at [s * 32 + L]; a lane walks its chunks one after another,
    # the last term of a chunk carries the chunk id (bit 20 set, id from bit 21); lanes are padded
    # with no-op terms (nu = 0) to the same number of steps
    seqs = [[[cterm[q] for q in range(cbeg[ch], cend[ch])] for ch in L] for L in lanes]
    il, ncdstep = _interleave(seqs, lambda t: t >> 8, lambda t, ch: t | (1 << 20) | (ch << 21),
                              [[ch for ch in L] for L in lanes], 0)
    hi["cd_sp_ptr"], hi["cd_il"] = spp, il

    # Jacobian, direct mass-action part: groups per (i, j), balanced over lanes
    groups: dict[tuple, list] = {}
    for p, r in enumerate(order):
        s = m32.slots[r]
        for rp, j in enumerate(s.C):
            for i in range(ns):
                if nu[i, r] != 0.0:
                    groups.setdefault((i, j), []).append((p << 12) | (rp << 8) | _nu8(nu[i, r]))
    keys = sorted(groups)
    lanes = _lpt([len(groups[k]) for k in keys])
    rs = nv if nv % 2 else nv + 1  # the solver's matrix row stride
    # interleaved int2 terms (x: slot | other reactant a << 10 | other reactant b << 17 | third-body
    # set << 24, none = 127; y: nu | target matrix offset << 8 | last-of-group << 20), so that a
    # term is decoded without looking up the slot's reactant word
    def jd_word(p, rp, nu8):
        s_ = m32.slots[order[p]]
        others = [c for o, c in enumerate(s_.C) if o != rp] + [NONE7, NONE7]
        mw = s_.M if s_.M >= 0 else NONE7
        return (p | (others[0] << 10) | (others[1] << 17) | (mw << 24), nu8)

    seqs = [[[jd_word(t >> 12, (t >> 8) & 15, t & 0xFF) for t in groups[keys[g]]] for g in L] for L in lanes]
    tgt_of = {g: keys[g][0] * rs + keys[g][1] for g in range(len(keys))}
    il, njdstep = _interleave(seqs, lambda w: w[0] & 1023, lambda w, g: (w[0], w[1] | (tgt_of[g] << 8) | (1 << 20)),
                              [list(L) for L in lanes], (0 | (NONE7 << 10) | (NONE7 << 17) | (NONE7 << 24), 0))
    if len(keys) and max(tgt_of.values()) >= 4096:
        raise ValueError("solver matrix too large for the packed Jacobian terms")
    ci["jd_il"] = [v for w in il for v in w]

    # Jacobian, third-body and falloff-[M] part: G[i][m] pairs
    pairs: dict[tuple, list] = {}
    for p, r in enumerate(order):
        s = m32.slots[r]
        src = []
        if s.M >= 0:
            src.append((s.M, 0))
        if s.kind == "falloff":
            src.append((s.M_fall, 1))
        for mm, kd in src:
            for i in range(ns):
                if nu[i, r] != 0.0:
                    pairs.setdefault((i, mm), []).append((p << 12) | (kd << 8) | _nu8(nu[i, r]))
    pkeys = sorted(pairs)
    lanes = _lpt([len(pairs[k]) for k in pkeys])
    ci["g_lane_ptr"], ci["g_lane_list"] = [0], []
    for L in lanes:
        ci["g_lane_list"] += L
        ci["g_lane_ptr"].append(len(ci["g_lane_list"]))
    ci["g_i"], ci["g_m"], ci["g_beg"], ci["g_end"], ci["g_term"] = [], [], [], [], []
    for k in pkeys:
        ci["g_i"].append(k[0]), ci["g_m"].append(k[1]), ci["g_beg"].append(len(ci["g_term"]))
        ci["g_term"] += pairs[k]
        ci["g_end"].append(len(ci["g_term"]))
    sizes = {"ns": ns, "nv": nv, "nslot": nslot, "nm": nm, "nfo": nfo, "nfc": nfc, "ncdchunk": len(cbeg),
             "njdgrp": len(keys), "ngpair": len(pkeys), "ncdstep": ncdstep, "njdstep": njdstep}
    return {"hd": hd, "hi": hi, "ci": ci, "sizes": sizes, "order": order}


SV_HD_KEYS = ("slot", "fo", "fc", "eff", "th", "wmol", "invw", "scal")
SV_HI_KEYS = ("slot", "fo", "fc", "cd_sp_ptr", "cd_il")
SV_CI_KEYS = ("jd_il", "g_lane_ptr", "g_lane_list", "g_i", "g_m", "g_beg", "g_end", "g_term")
SV_SIZE_KEYS = ("ns", "nv", "nslot", "nm", "nfo", "nfc", "ncdchunk", "njdgrp", "ngpair", "ncdstep", "njdstep")


def _interleave(seqs, slot_of, mark_last, ids, pad):
    """Per-lane term sequences -> one list with step s of lane L at [s * 32 + L].

    seqs[L] is lane L's list of groups (each a list of terms summed into one output); the last
    term of group g is replaced by mark_last(term, ids[L][g]). Terms within a group may be
    reordered: at every step each lane picks, from its current group, a term whose slot falls in a
    shared-memory bank (slot mod 16, 8-byte words) not yet used at this step by the other lanes of
    its half-warp, so that the 64-bit reads of the slot values are as conflict-free as possible.
    Lanes are padded to the same number of steps with `pad` (a no-op term)."""
    nsteps = max([sum(len(g) for g in L) for L in seqs] + [0])
    state = [[list(g) for g in L] for L in seqs]
    gi = [0] * 32
    out = [[pad] * 32 for _ in range(nsteps)]
    for st in range(nsteps):
        used = [set(), set()]
        for lane in range(32):
            L = state[lane] if lane < len(state) else []
            while gi[lane] < len(L) and not L[gi[lane]]:
                gi[lane] += 1
            if gi[lane] >= len(L):
                continue
            grp = L[gi[lane]]
            half = used[lane // 16]
            pick = 0
            for q, t in enumerate(grp):
                if slot_of(t) % 16 not in half:
                    pick = q
                    break
            t = grp.pop(pick)
            half.add(slot_of(t) % 16)
            if not grp:
                t = mark_last(t, ids[lane][gi[lane]])
            out[st][lane] = t
    return [t for row in out for t in row], nsteps


def solver_header(name: str) -> str:
    t = solver_tables(name)
    out = [f"// Generated by tiger_nga_b200/codegen.py: solver tables of mechanism {name}.",
           "#pragma once", '#include "solver_layout.h"', "namespace tng {"]

    def flat_int(src, keys):
        off, flat = [], []
        for k in keys:
            off.append(len(flat))
            flat += [int(x) for x in src[k]]
        return off, (flat or [0])

    hio, hif = flat_int(t["hi"], SV_HI_KEYS)
    cio, cif = flat_int(t["ci"], SV_CI_KEYS)
    hdo, hdf = [], [[], []]
    for k in SV_HD_KEYS:
        hdo.append(len(hdf[0]))
        for lm in (0, 1):
            hdf[lm] += t["hd"][k][lm]
    # keep the double block a multiple of 2 (16-byte staging granule)
    if len(hdf[0]) % 2:
        hdf[0].append(0.0), hdf[1].append(0.0)
    while len(hif) % 4:
        hif.append(0)
    out.append(f"static const double {name}_sv_hd[2][{len(hdf[0])}] = {{"
               + ", ".join("{" + ", ".join(_d(x) for x in hdf[lm]) + "}" for lm in (0, 1)) + "};")
    out.append(f"static const int {name}_sv_hi[{len(hif)}] = {{" + ", ".join(map(str, hif)) + "};")
    out.append(f"static const int {name}_sv_ci[{len(cif)}] = {{" + ", ".join(map(str, cif)) + "};")
    sz = ", ".join(str(t["sizes"][k]) for k in SV_SIZE_KEYS)
    out.append(f"static const SvLayout {name}_sv_layout = {{{{{sz}}}, {{{', '.join(map(str, hdo))}}}, "
               f"{{{', '.join(map(str, hio))}}}, {{{', '.join(map(str, cio))}}}, {len(hdf[0])}, {len(hif)}, "
               f"{len(cif)}}};")
    # the same layout as compile-time constants: the solver kernels are specialised on it
    def cfun(fname, vals):
        cases = " ".join(f"case {i}: return {v};" for i, v in enumerate(vals))
        return (f"  __host__ __device__ static constexpr int {fname}(int k) {{ switch (k) {{ {cases} default: return 0; }} }}")

    out.append(f"struct SvL_{name} {{")
    out.append(cfun("size", [t["sizes"][k] for k in SV_SIZE_KEYS]))
    out.append(cfun("hd", hdo))
    out.append(cfun("hi", hio))
    out.append(cfun("ci", cio))
    out.append(f"  static constexpr int nhd = {len(hdf[0])}, nhi = {len(hif)}, nci = {len(cif)};")
    out.append("};")
    out.append("}  // namespace tng")
    return "\n".join(out) + "\n"

if __name__ == "__main__":
    for p in write_all(sys.argv[1] if len(sys.argv) > 1 else "tiger_nga_b200/_build/gen"):
        print(p)
