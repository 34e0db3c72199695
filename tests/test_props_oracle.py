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


@pytest.mark.parametrize("mech", MECHS)
def test_wilke_rewrite_matches_the_reference_form(mech):
    """The transport kernel's algebra (tiger_nga_b200/codegen.py: Mech::transport / props_records)
    restated in NumPy against the reference's form (finitechem.f90:372-401): with q = W^1/4,
    phi_kj = A_kj (1 + sqrt(eta_k/eta_j) (W_j/W_k)^1/4)^2 = A_kj (1 + sig_k rho_j)^2, rho = q/sqrt(eta),
    sig = 1/rho, and row k's term u_k eta_k / sum_1 = u_k^2 q_k^2 / (w_k (u_k + A.u) + 2 v_k A.v + u_k A.w)
    with v = u rho, w = v rho. Also checks the sizes of the generated matrix and records."""
    from tiger_nga_b200 import codegen
    from tiger_nga_b200.mechanism import load

    m = load(mech)
    ns, W = m.ns, m.wmol
    g = codegen._Gen(mech)
    R, nrow = g.wilke_tile()
    assert nrow % R == 0 and nrow >= ns and R <= 13
    rng = np.random.default_rng(11)
    eta = 10 ** rng.uniform(-5.5, -4.0, ns)
    Y = rng.dirichlet(np.full(ns, 0.4))
    Y[0] = 0.0  # an absent species adds nothing
    u = Y / W
    # reference form (Y*W_mix/W factors cancel between sum_1 and sum_2)
    visc_ref = 0.0
    for k in range(ns):
        s1 = sum(u[j] * (1 / np.sqrt(8)) * (1 + W[k] / W[j]) ** -0.5 *
                 (1 + (eta[k] / eta[j]) ** 0.5 * (W[j] / W[k]) ** 0.25) ** 2 for j in range(ns) if j != k) + u[k]
        if Y[k] > 0:
            visc_ref += u[k] * eta[k] / s1
    # the kernel's form
    A = np.zeros((ns, ns))
    for k in range(ns):
        for j in range(ns):
            if j != k:
                A[k, j] = (1 / np.sqrt(8)) * (1 + W[k] / W[j]) ** -0.5
    q = W ** 0.25
    rho = q / np.sqrt(eta)
    v, w = u * rho, u * rho * rho
    a, b, c = A @ u, A @ v, A @ w
    visc = sum(u[k] ** 2 * q[k] ** 2 / (w[k] * (u[k] + a[k]) + 2 * b[k] * v[k] + c[k] * u[k])
               for k in range(ns) if u[k] > 0)
    assert abs(visc - visc_ref) <= 1e-13 * visc_ref
    # the generated constant tables hold the same numbers (reference literal kinds)
    src = g.props_records()
    assert f"{mech}_wilke[2][{nrow * ns}]" in src and f"{mech}_props_records[2][{ns * 19}]" in src
