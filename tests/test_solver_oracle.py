"""The CPU solver (the oracle's restatement of the implicit substep) against an independent
tight-tolerance integration, and its Jacobian against finite differences."""
import numpy as np
import pytest

from oracle.oracle import Oracle, solver_cfg
from tiger_nga_b200 import states
from tiger_nga_b200.mechanism import load

P = 101325.0
FUEL = {"hydrogen": "H2", "grimech30": "CH4", "dme39": "CH3OCH3"}


def batch(mech, n=64, seed=5):
    m = load(mech)
    minor = (1e-8, 1e-3) if mech == "hydrogen" else (1e-10, 1e-3)
    return states.chem_state(m, n, seed, FUEL[mech], grid=(n, 1, 1), minor=minor)[0]


@pytest.mark.parametrize("mech", ["hydrogen", "grimech30", "dme39"])
def test_jacobian_matches_finite_differences(mech):
    o = Oracle(mech)
    u = batch(mech, 8)[:, 3].copy()
    J = o.jacobian(u, P)
    Jfd = np.zeros_like(J)
    for j in range(len(u)):
        d = 1e-7 * max(abs(u[j]), 1e-12)
        du = np.zeros_like(u)
        du[j] = d
        Jfd[:, j] = (o.rhs(u + du, P) - o.rhs(u - du, P)) / (2 * d)
    scale = np.abs(Jfd).max(axis=1, keepdims=True) + 1e-300
    # exact except the falloff broadening's dependence on [M], which modified Newton tolerates
    assert np.max(np.abs(J - Jfd) / scale) < 1e-3


@pytest.mark.parametrize("mech,dt", [("hydrogen", 1e-6), ("hydrogen", 1e-5), ("grimech30", 1e-6)])
def test_substep_accuracy_vs_tight_radau(mech, dt):
    scipy_integrate = pytest.importorskip("scipy.integrate")
    o = Oracle(mech)
    sol = batch(mech, 16)
    out, st = o.substep_batch(sol, dt, P)
    assert np.all(st["status"] == 0)
    for i in range(0, 16, 4 if mech == "hydrogen" else 8):
        r = scipy_integrate.solve_ivp(lambda t, y: o.rhs(y, P), (0, dt), sol[:, i], method="Radau", rtol=1e-11,
                                      atol=1e-16, jac=lambda t, y: o.jacobian(y, P))
        ref = r.y[:, -1]
        Tr, To = ref[-1] / ref[:-1].sum(), out[-1, i] / out[:-1, i].sum()
        assert abs(To - Tr) / Tr < 1e-5
        assert np.max(np.abs(out[:-1, i] - ref[:-1])) / ref[:-1].sum() < 1e-6


def test_substep_edge_cases():
    o = Oracle("hydrogen")
    sol = batch("hydrogen", 4)
    out, st = o.substep_batch(sol, 0.0, P)  # dt = 0: unchanged
    assert np.array_equal(out, sol) and np.all(st["nst"] == 0)
    dts = np.array([1e-7, 1e-6, 0.0, 1e-5])  # per-cell dt
    out, st = o.substep_batch(sol, dts, P)
    assert st["nst"][2] == 0 and np.array_equal(out[:, 2], sol[:, 2]) and st["nst"][3] > st["nst"][0]
    bad = sol.copy()
    bad[3, 1] = np.nan  # non-finite input -> status 4, neighbours unaffected
    out, st = o.substep_batch(bad, 1e-6, P)
    assert st["status"][1] == 4 and st["status"][0] == 0 and st["status"][2] == 0
    out, st = o.substep_batch(sol, 1e-5, P, cfg=solver_cfg(max_steps=3))
    assert np.all(st["status"] == 1) and np.all(st["nst"] == 3)
