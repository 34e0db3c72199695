"""GPU parity of the batched right-hand side (finitechem_compute_rhs + PRODRATES) against the
CPU oracle and the golden reference fixtures, through the C-ABI.

Parity metric: production rates cancel near equilibrium, so the error of every rhs entry is
measured against its gross (cancellation-free) magnitude from the oracle,
``|d rhs_k| <= tol * gross_k`` with gross_k = W_k * sum_r |nu_kr W_r| and
gross_T = sum_k |h_k| gross_k / cp_mix.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle.oracle import Oracle  # noqa: E402
from tiger_nga_b200 import capi, states  # noqa: E402
from tiger_nga_b200.mechanism import load  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FUEL = {"hydrogen": "H2", "grimech30": "CH4", "dme39": "CH3OCH3"}
P = 101325.0
FP64_TOL = 1e-10  # FP64 mode: agreement with the reference arithmetic


def normwise(gpu, ref, gross):
    """max_k |gpu - ref| / gross, with gross floored at 1e-300 of the cell's largest entry."""
    gpu, ref, gross = (np.asarray(x) for x in (gpu, ref, gross))
    floor = np.maximum(gross.max(axis=0, keepdims=True) * 1e-300, 1e-300)
    return float(np.max(np.abs(gpu - ref) / np.maximum(gross, floor)))


def state(mech, n, seed=1):
    m = load(mech)
    sol, _ = states.chem_state(m, n, seed, FUEL[mech], grid=(n, 1, 1) if round(n ** (1 / 3)) ** 3 != n else None)
    return sol


def run_gpu(chem, sol, p=P):
    x = torch.from_numpy(sol).cuda()
    out = chem.compute_rhs(x, p)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def oracles():
    return {m: Oracle(m) for m in FUEL}


@pytest.mark.parametrize("mech", list(FUEL))
def test_fp64_matches_oracle(mech, oracles):
    sol = state(mech, 32 ** 3)
    chem = capi.FiniteChem(mech, "fp64")
    gpu = run_gpu(chem, sol)
    o = oracles[mech]
    ref = o.rhs_batch(sol, P)
    gross = o.rhs_gross_batch(sol, P)
    assert np.isfinite(gpu).all()
    assert normwise(gpu, ref, gross) <= FP64_TOL


@pytest.mark.parametrize("mech", list(FUEL))
def test_fp64_slot_rates_match_oracle(mech, oracles):
    """Every slot's rate W_r (the PRODRATES work array) agrees with the oracle."""
    sol = state(mech, 4099, seed=2)  # ragged against the 128-thread blocks: idle lanes must not store
    chem = capi.FiniteChem(mech, "fp64")
    x = torch.from_numpy(sol).cuda()
    _, rates = chem.compute_rhs_rates(x, P)
    torch.cuda.synchronize()
    W = rates.cpu().numpy()
    Wo = oracles[mech].rates_batch(sol, P)
    big = np.abs(Wo) > 1e-280
    rel = np.abs(W - Wo)[big] / np.abs(Wo)[big]
    assert rel.max() <= 1e-12, (rel.max(), np.unravel_index(np.argmax(np.where(big, np.abs(W - Wo) / np.maximum(np.abs(Wo), 1e-300), 0)), W.shape))


@pytest.mark.parametrize("mech", list(FUEL))
def test_fp64_matches_golden_reference_outputs(mech):
    """Inputs and outputs of the reference's own routines (transliterated Fortran)."""
    g = np.load(os.path.join(GOLDEN, f"{mech}_ref.npz"))
    chem = capi.FiniteChem(mech, "fp64")
    o = Oracle(mech)
    for p in np.unique(g["P"])[:4]:
        pass
    worst = 0.0
    for i in range(len(g["T"])):
        sol = np.ascontiguousarray(g["sol"][i][:, None])
        gpu = run_gpu(chem, sol, g["P"][i])[:, 0]
        gross = o.rhs_gross_batch(sol, g["P"][i])[:, 0]
        worst = max(worst, normwise(gpu[:, None], g["rhs"][i][:, None], gross[:, None]))
    assert worst <= FP64_TOL


@pytest.mark.parametrize("mech", ["grimech30", "dme39"])
def test_literal_mode_f64(mech):
    sol = state(mech, 4096, seed=3)
    chem = capi.FiniteChem(mech, "fp64", literal_mode="f64")
    o = Oracle(mech, "f64")
    assert normwise(run_gpu(chem, sol), o.rhs_batch(sol, P), o.rhs_gross_batch(sol, P)) <= FP64_TOL


@pytest.mark.parametrize("mech", list(FUEL))
def test_mixed_precision_error_bound(mech, oracles):
    """FP32 log-space rates with FP64 reverse exponents: error stated against the FP64 oracle."""
    sol = state(mech, 32 ** 3, seed=4)
    chem = capi.FiniteChem(mech, "mixed")
    gpu = run_gpu(chem, sol)
    o = oracles[mech]
    err = normwise(gpu, o.rhs_batch(sol, P), o.rhs_gross_batch(sol, P))
    assert np.isfinite(gpu).all()
    assert err <= 2e-4, err


def test_host_pointer_path_matches_device_path():
    sol = state("grimech30", 300_001, seed=5)  # several pipeline chunks, ragged tail
    chem = capi.FiniteChem("grimech30", "fp64")
    dev = run_gpu(chem, sol)
    host = chem.compute_rhs(sol, P)
    assert np.array_equal(dev, host)


@pytest.mark.parametrize("n", [1, 31, 33, 1000])
def test_ragged_and_strided_batches(n, oracles):
    sol = state("grimech30", n, seed=6)
    chem = capi.FiniteChem("grimech30", "fp64")
    ld = n + 13
    big = torch.zeros((37, ld), dtype=torch.float64, device="cuda")
    big[:, :n] = torch.from_numpy(sol).cuda()
    out = torch.full_like(big, 7.0)
    chem.compute_rhs(big[:, :n], P, out=out[:, :n])
    torch.cuda.synchronize()
    o = oracles["grimech30"]
    assert normwise(out[:, :n].cpu().numpy(), o.rhs_batch(sol, P), o.rhs_gross_batch(sol, P)) <= FP64_TOL
    assert torch.all(out[:, n:] == 7.0)  # nothing written past ncells


def test_empty_batch_and_bad_arguments():
    chem = capi.FiniteChem("hydrogen", "fp64")
    x = torch.zeros((10, 0), dtype=torch.float64, device="cuda")
    chem.compute_rhs(x, P)
    with pytest.raises(capi.ChemError):
        chem.compute_rhs(torch.ones((10, 4), dtype=torch.float64, device="cuda"), -1.0)


def test_range_switch_at_1000K(oracles):
    """COMPTHERMODATA switches ranges on T > 1000 strictly; T == 1000 uses the low range."""
    m = load("grimech30")
    o = oracles["grimech30"]
    Y = np.full(m.ns, 1.0 / m.ns)
    rho = 0.3
    cols = []
    for T in (1000.0, np.nextafter(1000.0, 0), np.nextafter(1000.0, 2000)):
        cols.append(np.concatenate([rho * Y, [rho * T]]))
    sol = np.ascontiguousarray(np.array(cols).T)
    chem = capi.FiniteChem("grimech30", "fp64")
    assert normwise(run_gpu(chem, sol), o.rhs_batch(sol, P), o.rhs_gross_batch(sol, P)) <= FP64_TOL


def test_full_size_grimech_properties(oracles):
    """128^3 cells: finite, mass-conserving to the molar-mass literals' rounding, and a random
    sample of 20k cells matches the oracle."""
    m = load("grimech30")
    sol, _ = states.ch4_cube(m, 128)
    chem = capi.FiniteChem("grimech30", "fp64")
    x = torch.from_numpy(sol).cuda()
    out = chem.compute_rhs(x, P)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(out).all())
    idx = np.random.default_rng(0).choice(sol.shape[1], 20000, replace=False)
    sub = np.ascontiguousarray(sol[:, idx])
    o = oracles["grimech30"]
    gross = o.rhs_gross_batch(sub, P)
    gpu = out[:, torch.from_numpy(idx).cuda()].cpu().numpy()
    assert normwise(gpu, o.rhs_batch(sub, P), gross) <= FP64_TOL
    mass = np.abs(gpu[:-1].sum(axis=0)) / gross[:-1].sum(axis=0)
    assert mass.max() < 1e-7
