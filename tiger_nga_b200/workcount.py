"""Algorithmic work per cell of the reference formulation, counted from the mechanism table.

These are the operation counts of the reference's own statements (not of the generated GPU
code, which does less): ``finitechem_compute_rhs`` (combustion/finitechem.f90:93-175) with
``PRODRATES`` (grimech30F.f90:4-2580), ``GETLINDRATECOEFF`` (:2583-2619) and
``COMPTHERMODATA`` (:2925-3516). Flops count + - * / once each; transcendentals (exp, log,
log10, pow) are counted separately, one each. Bytes are the state read and the rhs written,
(N+1) doubles each way.
"""
from __future__ import annotations

from .mechanism import Mechanism


def rhs_work(mech: Mechanism) -> dict:
    ns = mech.ns
    flops = 0
    exp = log = log10 = pw = 0
    # rho = sum(sol), Y = sol/rho, T = sol(N+1)/rho, cp_mix, conc, rhs_k, tmp, rhs_T
    flops += ns + ns + 1 + 2 * ns + ns + ns + 2 * ns + 1
    # COMPTHERMODATA: h 11 flops, cp 9 flops per species
    flops += 20 * ns
    # LT, RT
    log += 1
    flops += 1
    for terms in mech.third_body:
        flops += len(terms) - 1 + sum(1 for _, c in terms if c != 1.0)

    def arr(a):
        nonlocal flops, exp
        if a.n is None and a.E is None:
            return
        exp += 1
        flops += 1  # A * exp(...)
        flops += (1 if a.n is not None else 0) + (1 if a.E is not None else 0)
        flops += 1 if (a.n is not None and a.E is not None) else 0

    for s in mech.slots:
        if s.kind == "falloff":
            arr(s.k0)
            arr(s.kinf)
            for _ in s.fc:
                exp += 1
                flops += 3
            flops += len(s.fc) - 1
            # ntmp, cc (2 log10), Pr, log10(Pr), F, pow, final product
            log10 += 3
            pw += 1
            flops += 2 + 2 + 2 + 5 + 3 + 4
        else:
            arr(s.arr)
        flops += len(s.C) + (1 if s.M >= 0 else 0)
    for k in range(ns):
        nz = 0
        for r in range(mech.nslot):
            v = mech.nu[k, r]
            if v != 0.0:
                nz += 1
                flops += 1 if abs(v) != 1.0 else 0
        flops += max(nz - 1, 0)
    return {
        "flops": flops,
        "exp": exp,
        "log": log,
        "log10": log10,
        "pow": pw,
        "transcendentals": exp + log + log10 + pw,
        "bytes": 2 * (ns + 1) * 8,
    }
