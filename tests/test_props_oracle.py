"""The mixture-property oracle (finitechem_W / _density / _viscosity / _diffusivity,
combustion/finitechem.f90:65-74, :324-487) against the reference's own routines: the committed
golden fixtures (tests/golden/make_golden_props.py) and, where oracle/_ref was built, a fresh
random batch. Bit-exact: both sides are the same statement order under -ffp-contract=off."""
import os

import numpy as np
import pytest

from oracle.oracle import REF_LIB, Oracle, Reference

HERE = os.path.dirname(os.path.abspath(__file__))
MECHS = ("hydrogen", "grimech30", "dme39")


@pytest.mark.parametrize("mech", MECHS)
def test_props_oracle_matches_golden(mech):
    g = np.load(os.path.join(HERE, "golden", f"{mech}_props_ref.npz"))
    o = Oracle(mech)
    assert np.array_equal(o.mucoeff, g["mucoeff"]) and np.array_equal(o.koveps, g["koveps"])
    got = o.props_batch(g["Y"], g["T"], p_thermo=float(g["p"]), lewis=g["lewis"])
    for k in ("wmix", "rho", "visc", "diff"):
        assert np.array_equal(got[k], g[k], equal_nan=True), k


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("mech", MECHS)
def test_props_oracle_matches_reference_random(mech):
    o, r = Oracle(mech), Reference(mech)
    if getattr(r, "_pb", None) is None:
        pytest.skip("oracle/_ref predates the property routines")
    rng = np.random.default_rng(5)
    n = 512
    Y = rng.dirichlet(np.full(o.ns, 0.2), n).T.copy()
    Y[:, :20] *= -1e-4
    T = rng.uniform(10.0, 7000.0, n)
    a = o.props_batch(Y, T, p_thermo=3e5)
    b = r.props_batch(Y, T, p_thermo=3e5)
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_props_oracle_physics():
    """Sanity of the restated formulas on air-like mixtures: W_mix of N2/O2, rho from the ideal
    gas law, the viscosity of pure N2 near 1.8e-5 Pa s at 300 K, Lewis scaling."""
    o = Oracle("grimech30")
    sp = o.tab["species"]
    Y = np.zeros((o.ns, 2))
    Y[sp.index("N2"), 0] = 1.0
    Y[sp.index("N2"), 1], Y[sp.index("O2"), 1] = 0.767, 0.233
    T = np.array([300.0, 300.0])
    lew = np.full(o.ns, 2.0)
    out = o.props_batch(Y, T, p_thermo=101325.0, lewis=lew)
    assert abs(out["wmix"][0] - o.wmol[sp.index("N2")]) < 1e-12
    assert abs(out["wmix"][1] - 28.85) < 0.05
    assert np.allclose(out["rho"], 101325.0 * out["wmix"] / (8314.34 * T), rtol=1e-15)
    assert 1.5e-5 < out["visc"][0] < 2.1e-5
    assert np.allclose(out["diff"][:o.ns], out["diff"][o.ns] / 2.0, rtol=1e-15)
    assert 1.5e-5 < out["diff"][o.ns, 1] < 3.5e-5  # lambda/cp of air at 300 K [kg/(m s)]
