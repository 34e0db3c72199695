"""Regenerate the golden rate fixtures from the reference's own mechanism routines.

Runs ``oracle/_ref/libref_mech.so`` -- the reference's Fortran PRODRATES / COMPTHERMODATA /
GETMOLARMASS transliterated statement by statement to C by ``oracle/f90_to_c.py`` (it needs
the reference tree to build) -- on seeded inputs, and stores inputs and outputs as
``tests/golden/<mechanism>_ref.npz``. The fixtures pin the table-driven oracle on machines
where the reference tree is absent.

    python oracle/f90_to_c.py <reference>/combustion && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402


def cases(ns, seed, n=32):
    rng = np.random.default_rng(seed)
    Ts, Cs, Ps = [], [], []
    for i in range(n):
        T = rng.uniform(280.0, 3000.0)
        if i == 0:
            T = 1000.0  # the range switch (T.GT.1000 is strict)
        elif i == 1:
            T = np.nextafter(1000.0, 2000.0)
        elif i == 2:
            T = 300.0
        C = 10.0 ** rng.uniform(-14.0, -1.0, ns)
        if i % 6 == 3:
            C[rng.integers(0, ns, 3)] = 0.0  # absent species
        if i == 4:
            C[:] = 0.0  # all-zero concentrations: third-body sums 0, falloff uses P/(RT)
        Ts.append(T), Cs.append(C), Ps.append(101325.0 * rng.uniform(0.2, 5.0))
    return np.array(Cs), np.array(Ts), np.array(Ps)


def main():
    for name, seed in (("hydrogen", 11), ("grimech30", 12), ("dme39", 13)):
        ref = Reference(name)
        C, T, P = cases(ref.ns, seed)
        cd, W, K, M, h, cp, sol, rhs = ([] for _ in range(8))
        for c, t, p in zip(C, T, P):
            a, b, k, m = ref.prodrates(c, t, p)
            cd.append(a), W.append(b), K.append(k), M.append(m)
            hh, cc = ref.thermo(t)
            h.append(hh), cp.append(cc)
            s = np.concatenate([c * ref.wmol, [np.sum(c * ref.wmol) * t]])
            if s[:-1].sum() == 0.0:
                s[:-1] = ref.wmol * 1e-3
                s[-1] = s[:-1].sum() * t
            sol.append(s)
            rhs.append(ref.rhs(s, p))
        out = os.path.join(HERE, f"{name}_ref.npz")
        np.savez_compressed(out, C=C, T=T, P=P, cdot=np.array(cd), W=np.array(W), K=np.array(K), M=np.array(M),
                            h=np.array(h), cp=np.array(cp), wmol=ref.wmol, sol=np.array(sol), rhs=np.array(rhs))
        print(out, os.path.getsize(out))


if __name__ == "__main__":
    main()
