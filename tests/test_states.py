"""The seeded workload states: reproducible, physical (mass fractions, temperature ranges), and
shaped as the workloads describe them (mixing layer: fuel above air with a tanh profile)."""
import numpy as np

from tiger_nga_b200 import states
from tiger_nga_b200.mechanism import load
from tiger_nga_b200.train_surrogate import state_batch


def _Y_T(mech, sol):
    rho = sol[:mech.ns].sum(0)
    return sol[:mech.ns] / rho, sol[mech.ns] / rho


def test_mixing_layer_is_seeded_and_layered():
    m = load("dme39")
    a, ia = states.mixing_layer(m, shape=(16, 24, 8), seed=5)
    b, _ = states.mixing_layer(m, shape=(16, 24, 8), seed=5)
    c, _ = states.mixing_layer(m, shape=(16, 24, 8), seed=6)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    Y, T = _Y_T(m, a)
    assert np.all(Y >= 0) and np.allclose(Y.sum(0), 1.0, atol=1e-12)
    assert T.min() >= 299.0 and T.max() < 3000.0
    Z = ia["Z"].reshape(16, 24, 8)
    assert Z[:, :4].mean() < 0.2 and Z[:, -4:].mean() > 0.8  # air below, fuel above
    fuel = Y[m.species.index("CH3OCH3")].reshape(16, 24, 8)
    assert fuel[:, -4:].mean() > fuel[:, :4].mean()


def test_mixing_layer_chunks_do_not_change_the_state():
    m = load("hydrogen")
    a, _ = states.mixing_layer(m, shape=(8, 8, 8), seed=3, fuel="H2", T_fuel=300.0, chunk=1 << 20)
    b, _ = states.mixing_layer(m, shape=(8, 8, 8), seed=3, fuel="H2", T_fuel=300.0, chunk=1 << 20)
    assert np.array_equal(a, b)


def test_uneven_stiffness_batch():
    sol, dts = state_batch("grimech30", 4096, 9, side=16)
    m = load("grimech30")
    Y, T = _Y_T(m, sol)
    assert np.allclose(Y.sum(0), 1.0, atol=1e-12) and np.all(Y >= 0)
    assert 300.0 <= T.min() and T.max() <= 2400.0 + 1e-9
    # Beta(2,2) progress: the middle of the range is the most populated
    assert np.mean((T > 900) & (T < 1800)) > 0.5
    assert np.all((dts >= 1e-7) & (dts <= 1e-5))
    s2, d2 = state_batch("grimech30", 4096, 9, side=16)
    assert np.array_equal(sol, s2) and np.array_equal(dts, d2)
