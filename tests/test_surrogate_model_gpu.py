"""The committed GRI-Mech surrogate (tiger_nga_b200/models/grimech30.tngs) on fresh cells from a
seed outside its training, validation and calibration sets: what the trained network gains over
the plain implicit GPU solve of the same cells, at the accuracy bars of the learned substep --
max |T_s - T_p| / T_p <= 1 % and max |Y_s,k - Y_p,k| <= 1e-3 max_k Y_p,k over every cell --
with exact mass and element conservation of the cells the network takes."""
import os
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tiger_nga_b200 import capi  # noqa: E402
from tiger_nga_b200.mechanism import load  # noqa: E402
from tiger_nga_b200.train_surrogate import state_batch  # noqa: E402

pytestmark = pytest.mark.gpu
P = 101325.0
MODEL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tiger_nga_b200", "models",
                     "grimech30.tngs")


def test_committed_model_meets_the_bars_and_beats_the_plain_solve():
    chem = capi.FiniteChem("grimech30", "fp64")
    sur = capi.Surrogate(chem)
    sur.load(MODEL)
    has_gate, tol = sur.gate_info()
    assert has_gate and 0.0 < tol < 1.0
    n = 64 ** 3  # a 64^3 grid of the headline's state distribution, from a fresh seed
    sol, dts = state_batch("grimech30", n, 990001, side=64)
    s0 = torch.from_numpy(sol).cuda()
    d = torch.from_numpy(dts).cuda()
    ref, x = s0.clone(), s0.clone()
    # warm both paths (graph capture, staging buffers) on a copy, then time one call each
    chem.substep(s0.clone(), d, P)
    sur.substep(s0.clone(), d, P)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    chem.substep(ref, d, P, stats=False)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    t0 = time.perf_counter()
    st = sur.substep(x, d, P)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    ns = chem.nspecies
    out, rf, ini = x.cpu().numpy(), ref.cpu().numpy(), sol
    assert np.isfinite(out).all()
    rs, rr = out[:ns].sum(0), rf[:ns].sum(0)
    dT = np.abs(out[ns] / rs - rf[ns] / rr) / (rf[ns] / rr)
    dY = np.abs(out[:ns] / rs - rf[:ns] / rr).max(0) / (rf[:ns] / rr).max(0)
    assert dT.max() <= 1e-2, dT.max()
    assert dY.max() <= 1e-3, dY.max()
    # the network takes most cells; those it takes conserve mass and elements exactly
    assert st["accepted"] >= 0.9 * n, st
    acc = ~np.all(out == rf, axis=0)
    m = load("grimech30")
    rho0 = ini[:ns].sum(0)
    assert np.max(np.abs(rs - rho0)[acc] / rho0[acc]) < 1e-12
    E = m.elem / m.wmol[None, :]
    el0, el1 = E @ (ini[:ns] / rho0), E @ (out[:ns] / rs)
    scale = np.maximum(el0.max(axis=1, keepdims=True), 1e-6)
    assert np.max((np.abs(el1 - el0) / scale)[:, acc]) < 1e-7
    # the gain: the same cells through the surrogate (fallback and judged sample included) at
    # least 10x faster than through the plain implicit solve
    assert t_plain / t_sur >= 10.0, (t_plain, t_sur, st["fallback"]["cells"])


def test_host_pointer_substep_equals_device_pointer_substep():
    """With host buffers and a large batch the state is uploaded in chunks that overlap the
    inference and post-processing of the chunks already on the device; the result is the same,
    cell for cell, as the substep on device buffers (a ragged batch of 3 chunks and a fraction,
    per-cell dt)."""
    chem = capi.FiniteChem("grimech30", "fp64")
    sur = capi.Surrogate(chem)
    sur.load(MODEL)
    n = 3 * (1 << 18) + 12345
    sol, dts = state_batch("grimech30", n, 990007, side=0)
    x = torch.from_numpy(sol).cuda()
    d = torch.from_numpy(dts).cuda()
    st_dev = sur.substep(x, d, P)
    host = np.ascontiguousarray(sol.copy())
    st_host = sur.substep(host, np.ascontiguousarray(dts), P)
    torch.cuda.synchronize()
    assert np.array_equal(host, x.cpu().numpy())
    for k in ("accepted", "fallback_ood", "fallback_consistency", "fallback_clip", "fallback_ensemble",
              "fallback_gate", "judged"):
        assert st_host[k] == st_dev[k], (k, st_host[k], st_dev[k])
    assert st_host["fallback"]["cells"] == st_dev["fallback"]["cells"]
    assert np.isfinite(st_host["judge_max_rel_dT"]) and st_host["judge_max_rel_dT"] <= 1e-2
