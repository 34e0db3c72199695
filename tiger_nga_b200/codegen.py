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
                    o.append(f"    if (DUMP) dump[{r}LL * dld] = w;")
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
                o.append(f"    if (DUMP) dump[{r}LL * dld] = w;")
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

    def header(self) -> str:
        m32, m64 = self.m32, self.m64
        cls = f"Mech_{self.name}"
        out = [f"// Generated from tiger_nga_b200/mechanisms/{self.name}.json by tiger_nga_b200/codegen.py.",
               "// Do not edit: regenerate with tiger_nga_b200.build.",
               "#pragma once",
               '#include "tng_device.cuh"',
               "namespace tng {",
               f"struct {cls} {{",
               f"  static constexpr int NS = {self.ns};",
               f"  static constexpr int NSLOT = {self.nslot};",
               f"  static constexpr int NM = {self.nm};",
               f'  static constexpr const char* NAME = "{self.name}";']
        out.append(self.rhs("fp64", dump=True))
        out.append(self.rhs("mixed", dump=True))
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

SV_SCALARS = ("rgas", "tmid", "troe_n0", "troe_n1", "troe_c0", "troe_c1", "troe_d", "lnkmin", "inv_ln10")


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


def solver_tables(name: str) -> dict:
    """Flat double/int tables for one mechanism: doubles per literal mode, ints shared."""
    g = _Gen(name)
    m32, m64 = g.m32, g.m64
    ns, nslot, nm = g.ns, g.nslot, g.nm
    nv = ns + 1
    ints: dict[str, list[int]] = {}
    dbl: dict[str, list[list[float]]] = {}

    def D(key, v32, v64):
        dbl[key] = [list(map(float, v32)), list(map(float, v64))]

    # slots
    flags, A, lnA, nn, EE, reac, mw, fo = ([], [], [], [], [], [], [], [])
    A6, lnA6, nn6, EE6 = [], [], [], []
    fos = []
    for s32, s64 in zip(m32.slots, m64.slots):
        reac.extend((s32.C + [-1, -1, -1])[:3])
        mw.append(s32.M)
        if s32.kind == "falloff":
            flags.append(1)
            fo.append(len(fos))
            fos.append((s32, s64))
            A.append(0.0), lnA.append(0.0), nn.append(0.0), EE.append(0.0)
            A6.append(0.0), lnA6.append(0.0), nn6.append(0.0), EE6.append(0.0)
            continue
        a, b = s32.arr, s64.arr
        f = (2 if a.n is not None else 0) | (4 if a.E is not None else 0)
        if f == 0:
            f = 8
        flags.append(f)
        fo.append(-1)
        A.append(a.A), A6.append(b.A)
        lnA.append(math.log(a.A)), lnA6.append(math.log(b.A))
        nn.append(a.n or 0.0), nn6.append(b.n or 0.0)
        EE.append(a.E or 0.0), EE6.append(b.E or 0.0)
    ints["slot_flags"], ints["slot_reac"], ints["slot_mw"], ints["slot_fo"] = flags, reac, mw, fo
    D("slot_A", A, A6), D("slot_lnA", lnA, lnA6), D("slot_n", nn, nn6), D("slot_E", EE, EE6)

    # falloff and F_cent expressions
    fc_ids: dict[tuple, int] = {}
    fc_terms32: list[list] = []
    fc_terms64: list[list] = []
    fo_flags, fo_fc, fo_m = [], [], []
    fo_d32, fo_d64 = [], []
    for s32, s64 in fos:
        row32, row64, fl = [], [], []
        for a, b in ((s32.k0, s64.k0), (s32.kinf, s64.kinf)):
            fl.append((2 if a.n is not None else 0) | (4 if a.E is not None else 0))
            row32 += [math.log(a.A), a.n or 0.0, a.E or 0.0]
            row64 += [math.log(b.A), b.n or 0.0, b.E or 0.0]
        fo_flags += fl
        fo_d32 += row32
        fo_d64 += row64
        fo_m.append(s32.M_fall)
        key = s32.fc_key
        if key == ((1.0, 1, 0.0),):
            fo_fc.append(-1)
            continue
        if key not in fc_ids:
            fc_ids[key] = len(fc_ids)
            t32, t64 = [], []
            for (a, form, x), (a6, _, x6) in zip(s32.fc, s64.fc):
                if form == 0 and x <= 1e-20:
                    continue
                if form == 1 and x >= 1e20:
                    continue
                if (form == 0 and x >= 1e20) or (form == 1 and x == 0.0):
                    t32.append((2, a, 0.0)), t64.append((2, a6, 0.0))
                elif form == 0:
                    t32.append((0, a, 1.0 / x)), t64.append((0, a6, 1.0 / x6))
                else:
                    t32.append((1, a, x)), t64.append((1, a6, x6))
            assert 1 <= len(t32) <= 3
            fc_terms32.append(t32)
            fc_terms64.append(t64)
        fo_fc.append(fc_ids[key])
    nfo, nfc = len(fos), len(fc_ids)
    ints["fo_flags"], ints["fo_fc"], ints["fo_m"] = fo_flags, fo_fc, fo_m
    D("fo_par", fo_d32, fo_d64)
    fcf, fca32, fcc32, fca64, fcc64 = [], [], [], [], []
    for t32, t64 in zip(fc_terms32, fc_terms64):
        for i in range(3):
            if i < len(t32):
                fcf.append(t32[i][0]), fca32.append(t32[i][1]), fcc32.append(t32[i][2])
                fca64.append(t64[i][1]), fcc64.append(t64[i][2])
            else:
                fcf.append(-1), fca32.append(0.0), fcc32.append(0.0), fca64.append(0.0), fcc64.append(0.0)
    ints["fc_form"] = fcf
    D("fc_a", fca32, fca64), D("fc_c", fcc32, fcc64)

    # third-body sums (table order) and dense efficiencies
    tb_ptr, tb_sp, tbc32, tbc64 = [0], [], [], []
    eff32 = np.zeros((max(nm, 1), ns))
    eff64 = np.zeros((max(nm, 1), ns))
    for j, (t32, t64) in enumerate(zip(m32.third_body, m64.third_body)):
        for (s_, c), (_, c6) in zip(t32, t64):
            tb_sp.append(s_), tbc32.append(c), tbc64.append(c6)
            eff32[j, s_] += c
            eff64[j, s_] += c6
        tb_ptr.append(len(tb_sp))
    ints["tb_ptr"], ints["tb_sp"] = tb_ptr, tb_sp
    D("tb_coef", tbc32, tbc64), D("eff", eff32.reshape(-1), eff64.reshape(-1))

    # production rates: species rows split into chunks, chunks balanced over lanes
    total = int((m32.nu != 0).sum())
    chunk = max(8, -(-total // 32))
    cd_chunk_sp, cd_chunk_beg, cd_chunk_end, cd_slot, cdn32, cdn64, cd_sp_ptr = [], [], [], [], [], [], [0]
    for k in range(ns):
        rs = [r for r in range(nslot) if m32.nu[k, r] != 0.0 or m64.nu[k, r] != 0.0]
        for b in range(0, len(rs), chunk):
            cd_chunk_sp.append(k)
            cd_chunk_beg.append(len(cd_slot))
            for r in rs[b:b + chunk]:
                cd_slot.append(r), cdn32.append(m32.nu[k, r]), cdn64.append(m64.nu[k, r])
            cd_chunk_end.append(len(cd_slot))
        cd_sp_ptr.append(len(cd_chunk_sp))
    lanes = _lpt([e - b for b, e in zip(cd_chunk_beg, cd_chunk_end)])
    ints["cd_lane_ptr"] = [0]
    ints["cd_lane_list"] = []
    for L in lanes:
        ints["cd_lane_list"] += L
        ints["cd_lane_ptr"].append(len(ints["cd_lane_list"]))
    ints["cd_chunk_beg"], ints["cd_chunk_end"], ints["cd_slot"], ints["cd_sp_ptr"] = (
        cd_chunk_beg, cd_chunk_end, cd_slot, cd_sp_ptr)
    D("cd_nu", cdn32, cdn64)

    # Jacobian, direct mass-action part: groups per (i, j), balanced over lanes
    groups: dict[tuple, list] = {}
    for s in m32.slots:
        r = s.index
        for pidx, j in enumerate(s.C):
            for i in range(ns):
                if m32.nu[i, r] != 0.0 or m64.nu[i, r] != 0.0:
                    groups.setdefault((i, j), []).append((r, pidx, m32.nu[i, r], m64.nu[i, r]))
    keys = sorted(groups)
    lanes = _lpt([len(groups[k]) for k in keys])
    jd_tgt, jd_beg, jd_end, jd_slot, jd_pos, jdn32, jdn64 = [], [], [], [], [], [], []
    for k in keys:
        jd_tgt.append(k[0] * nv + k[1])
        jd_beg.append(len(jd_slot))
        for r, pidx, a, b in groups[k]:
            jd_slot.append(r), jd_pos.append(pidx), jdn32.append(a), jdn64.append(b)
        jd_end.append(len(jd_slot))
    ints["jd_lane_ptr"], ints["jd_lane_list"] = [0], []
    for L in lanes:
        ints["jd_lane_list"] += L
        ints["jd_lane_ptr"].append(len(ints["jd_lane_list"]))
    ints["jd_tgt"], ints["jd_beg"], ints["jd_end"], ints["jd_slot"], ints["jd_pos"] = jd_tgt, jd_beg, jd_end, jd_slot, jd_pos
    D("jd_nu", jdn32, jdn64)

    # Jacobian, third-body and falloff-[M] part: G[i][m] pairs
    pairs: dict[tuple, list] = {}
    for s in m32.slots:
        r = s.index
        src = []
        if s.M >= 0:
            src.append((s.M, 0))
        if s.kind == "falloff":
            src.append((s.M_fall, 1))
        for mm, kind in src:
            for i in range(ns):
                if m32.nu[i, r] != 0.0 or m64.nu[i, r] != 0.0:
                    pairs.setdefault((i, mm), []).append((r, kind, m32.nu[i, r], m64.nu[i, r]))
    pkeys = sorted(pairs)
    lanes = _lpt([len(pairs[k]) for k in pkeys])
    g_i, g_m, g_beg, g_end, g_slot, g_kind, gn32, gn64 = [], [], [], [], [], [], [], []
    for k in pkeys:
        g_i.append(k[0]), g_m.append(k[1]), g_beg.append(len(g_slot))
        for r, kind, a, b in pairs[k]:
            g_slot.append(r), g_kind.append(kind), gn32.append(a), gn64.append(b)
        g_end.append(len(g_slot))
    ints["g_lane_ptr"], ints["g_lane_list"] = [0], []
    for L in lanes:
        ints["g_lane_list"] += L
        ints["g_lane_ptr"].append(len(ints["g_lane_list"]))
    ints["g_i"], ints["g_m"], ints["g_beg"], ints["g_end"], ints["g_slot"], ints["g_kind"] = (
        g_i, g_m, g_beg, g_end, g_slot, g_kind)
    D("g_nu", gn32, gn64)

    # thermo and molar masses
    D("th_hi", m32.th_hi.reshape(-1), m64.th_hi.reshape(-1))
    D("th_lo", m32.th_lo.reshape(-1), m64.th_lo.reshape(-1))
    D("wmol", m32.wmol, m64.wmol)
    D("invw", 1.0 / m32.wmol, 1.0 / m64.wmol)
    sc = []
    for mm in (m32, m64):
        t = mm.troe
        sc.append([mm.rgas, mm.tmid, t["c_n0"], t["c_n1"], t["c_c0"], t["c_c1"], t["c_d"], math.log(t["kmin"]),
                   INV_LN10])
    dbl["scal"] = sc
    sizes = {"ns": ns, "nv": nv, "nslot": nslot, "nm": nm, "nfo": nfo, "nfc": nfc, "ncdchunk": len(cd_chunk_beg),
             "njdgrp": len(jd_tgt), "ngpair": len(g_i)}
    return {"ints": ints, "dbl": dbl, "sizes": sizes}


SV_INT_KEYS = ("slot_flags", "slot_reac", "slot_mw", "slot_fo", "fo_flags", "fo_fc", "fo_m", "fc_form", "tb_ptr",
               "tb_sp", "cd_lane_ptr", "cd_lane_list", "cd_chunk_beg", "cd_chunk_end", "cd_slot", "cd_sp_ptr",
               "jd_lane_ptr", "jd_lane_list", "jd_tgt", "jd_beg", "jd_end", "jd_slot", "jd_pos",
               "g_lane_ptr", "g_lane_list", "g_i", "g_m", "g_beg", "g_end", "g_slot", "g_kind")
SV_DBL_KEYS = ("slot_A", "slot_lnA", "slot_n", "slot_E", "fo_par", "fc_a", "fc_c", "tb_coef", "eff", "cd_nu", "jd_nu",
               "g_nu", "th_hi", "th_lo", "wmol", "invw", "scal")
SV_SIZE_KEYS = ("ns", "nv", "nslot", "nm", "nfo", "nfc", "ncdchunk", "njdgrp", "ngpair")


def solver_header(name: str) -> str:
    t = solver_tables(name)
    out = [f"// Generated by tiger_nga_b200/codegen.py: solver tables of mechanism {name}.",
           "#pragma once", '#include "solver_layout.h"', "namespace tng {"]
    ioff, iflat = [], []
    for k in SV_INT_KEYS:
        ioff.append(len(iflat))
        iflat += [int(x) for x in t["ints"][k]]
    doff, dflat = [], [[], []]
    for k in SV_DBL_KEYS:
        doff.append(len(dflat[0]))
        for lm in (0, 1):
            dflat[lm] += t["dbl"][k][lm]
    iflat = iflat or [0]
    out.append(f"static const int {name}_sv_int[{len(iflat)}] = {{" + ", ".join(map(str, iflat)) + "};")
    out.append(f"static const double {name}_sv_dbl[2][{len(dflat[0])}] = {{"
               + ", ".join("{" + ", ".join(_d(x) for x in dflat[lm]) + "}" for lm in (0, 1)) + "};")
    sz = ", ".join(str(t["sizes"][k]) for k in SV_SIZE_KEYS)
    out.append(f"static const SvLayout {name}_sv_layout = {{{{{sz}}}, {{{', '.join(map(str, ioff))}}}, "
               f"{{{', '.join(map(str, doff))}}}, {len(iflat)}, {len(dflat[0])}}};")
    out.append("}  // namespace tng")
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    for p in write_all(sys.argv[1] if len(sys.argv) > 1 else "tiger_nga_b200/_build/gen"):
        print(p)
