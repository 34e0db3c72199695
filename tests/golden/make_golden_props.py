"""Regenerate the golden mixture-property fixtures from the reference's own routines.

Runs ``oracle/_ref/libref_mech.so`` -- the reference's GETMOLARMASS / GETMUCOEFF / GETKOVEREPS /
COMPTHERMODATA transliterated statement by statement to C by ``oracle/f90_to_c.py``, under the
statement-order restatement of finitechem_W / _density / _viscosity / _diffusivity
(combustion/finitechem.f90:65-74, :324-487) -- on seeded cells, and stores inputs and outputs
as ``tests/golden/<mechanism>_props_ref.npz``. They pin the table-driven oracle where the
reference tree is absent.

    python oracle/f90_to_c.py <reference>/combustion && python tests/golden/make_golden_props.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402


def cells(ns, seed, n=32):
    rng = np.random.default_rng(seed)
    Y = rng.dirichlet(np.full(ns, 0.3), n).T.copy()
    T = rng.uniform(250.0, 3200.0, n)
    T[0], T[1], T[2], T[3] = 1000.0, np.nextafter(1000.0, 2000.0), 20.0, 6500.0  # range switch, both clips
    Y[:, 4] = 0.0
    Y[0, 4] = 1.0  # a pure species
    Y[rng.integers(0, ns, 3), 5] = -1e-9  # slightly negative mass fractions
    Y[:, 6] *= 1.3  # sum above one (the W_mix clip)
    return Y, T


def main():
    for name, seed in (("hydrogen", 21), ("grimech30", 22), ("dme39", 23)):
        ref = Reference(name)
        Y, T = cells(ref.ns, seed)
        lewis = np.random.default_rng(seed + 100).uniform(0.7, 1.6, ref.ns)
        p = 101325.0 * 1.7
        out = ref.props_batch(Y, T, p_thermo=p, lewis=lewis)
        np.savez_compressed(os.path.join(HERE, f"{name}_props_ref.npz"), Y=Y, T=T, lewis=lewis, p=p,
                            mucoeff=ref.mucoeff, koveps=ref.koveps, **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
