"""The project's autotuner: it times the candidate launch configurations on the caller's cells,
keeps the fastest, and changes nothing but the speed (per-cell results are identical)."""
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tiger_nga_b200 import capi  # noqa: E402
from tiger_nga_b200.train_surrogate import state_batch  # noqa: E402

pytestmark = pytest.mark.gpu
P = 101325.0


def test_substep_autotune_keeps_results_and_caches(tmp_path):
    sol, dts = state_batch("grimech30", 2048, 41, side=0)
    x0 = torch.from_numpy(sol).cuda()
    d = torch.from_numpy(dts).cuda()
    chem = capi.FiniteChem("grimech30", "fp64")
    ref = x0.clone()
    chem.substep(ref, d, P)
    cache = str(tmp_path / "tune.json")
    r = chem.autotune(x0, d, P, kind="substep", sample=512, cache=cache)
    assert len(r["candidates"]) == 12 and all(ms > 0 for _, _, ms in r["candidates"])
    assert tuple(r["best"]) in {(a, b) for a, b, _ in r["candidates"]}
    got = x0.clone()
    chem.substep(got, d, P)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)  # the choice changes the speed only
    stored = json.load(open(cache))
    chem2 = capi.FiniteChem("grimech30", "fp64")
    r2 = chem2.autotune(x0, d, P, kind="substep", cache=cache)  # applied from the cache, no timing
    assert tuple(r2["best"]) == tuple(r["best"]) and len(stored) == 1
    a, b = r["best"]
    assert (chem2.cfg.solver_warps, chem2.cfg.solver_occupancy, chem2.cfg.pass_budget) == \
        ((8, 2) if a == 16 else (a, 1)) + (b,)


def test_rates_autotune_keeps_results():
    sol, _ = state_batch("grimech30", 65536, 42, side=0)
    x = torch.from_numpy(sol).cuda()
    chem = capi.FiniteChem("grimech30", "fp64")
    ref = chem.compute_rhs(x, P).clone()
    r = chem.autotune(x, None, P, kind="rates")
    assert len(r["candidates"]) == 9
    got = chem.compute_rhs(x, P)
    torch.cuda.synchronize()
    scale = ref.abs().amax(dim=1, keepdim=True) + 1e-300
    # variants differ only in scheduling (barriers, register caps), not in the arithmetic
    assert float(((got - ref).abs() / scale).max()) <= 1e-13
