"""The CPU oracle against the reference: golden fixtures (always) and the transliterated
reference library (where it was built from the reference tree)."""
import os

import numpy as np
import pytest

from oracle.oracle import REF_LIB, Oracle, Reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
MECHS = ["hydrogen", "grimech30", "dme39"]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.where(d == 0, 0.0, d / s)))


@pytest.mark.parametrize("mech", MECHS)
def test_oracle_reproduces_golden(mech):
    g = np.load(os.path.join(GOLDEN, f"{mech}_ref.npz"))
    o = Oracle(mech)
    assert np.array_equal(o.wmol, g["wmol"])
    worst = 0.0
    for i in range(len(g["T"])):
        cd, W, K, M = o.prodrates(g["C"][i], g["T"][i], g["P"][i])
        h, cp = o.thermo(g["T"][i])
        for a, b in ((cd, g["cdot"][i]), (W, g["W"][i]), (K, g["K"][i]), (M, g["M"][i]), (h, g["h"][i]),
                     (cp, g["cp"][i]), (o.rhs(g["sol"][i], g["P"][i]), g["rhs"][i])):
            worst = max(worst, _rel(a, b))
    # same operation order and literal kinds as the reference; only libm could differ
    assert worst <= 1e-14, worst


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("mech", MECHS)
def test_oracle_bit_exact_vs_transliterated_reference(mech):
    o, r = Oracle(mech), Reference(mech)
    rng = np.random.default_rng(5)
    for _ in range(100):
        T = rng.uniform(250, 3200)
        C = 10 ** rng.uniform(-15, 0, o.ns)
        P = 101325 * rng.uniform(0.1, 10)
        for a, b in zip(o.prodrates(C, T, P), r.prodrates(C, T, P)):
            assert np.array_equal(a, b)
        sol = np.concatenate([C * o.wmol, [np.sum(C * o.wmol) * T]])
        assert np.array_equal(o.rhs(sol, P), r.rhs(sol, P))


def test_literal_kind_matters():
    """Default-real literals are float32 in the reference build: reading them as doubles moves
    K(R1F) of the H2 mechanism by ~1e-7 relative at 1500 K -- far above 1e-10."""
    o32, o64 = Oracle("hydrogen", "f32"), Oracle("hydrogen", "f64")
    C = np.full(9, 1e-3)
    k32 = o32.prodrates(C, 1500.0, 101325.0)[2][0]
    k64 = o64.prodrates(C, 1500.0, 101325.0)[2][0]
    assert 1e-8 < abs(k32 - k64) / k64 < 1e-6


@pytest.mark.parametrize("mech,mode,tol", [("grimech30", "f32", 1e-7), ("grimech30", "f64", 1e-12),
                                           ("dme39", "f32", 1e-7), ("hydrogen", "f64", 1e-12)])
def test_mass_conservation(mech, mode, tol):
    """sum_k cdot_k W_k = 0 up to the molar-mass literals' rounding (float32 in the reference)."""
    from tiger_nga_b200 import states
    from tiger_nga_b200.mechanism import load

    m = load(mech, mode)
    fuel = {"grimech30": "CH4", "dme39": "CH3OCH3", "hydrogen": "H2"}[mech]
    sol, _ = states.chem_state(m, 512, 3, fuel, grid=(8, 8, 8))
    o = Oracle(mech, mode)
    r = o.rhs_batch(sol, 101325.0)
    g = o.rhs_gross_batch(sol, 101325.0)
    assert np.max(np.abs(r[:-1].sum(0)) / g[:-1].sum(0)) < tol
