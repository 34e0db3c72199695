"""tng_substep_batch_static (scratch in a static device array, nothing allocated per call)
against tng_substep_batch on the same cells, on two calls in a row (the second call checks
that the state which must start at zero is cleared again)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tiger_nga_b200 import capi, states  # noqa: E402
from tiger_nga_b200.mechanism import load  # noqa: E402

pytestmark = pytest.mark.gpu
P = 101325.0


@pytest.mark.parametrize("mech,fuel", [("hydrogen", "H2"), ("grimech30", "CH4")])
def test_static_scratch_matches_batch_on_consecutive_calls(mech, fuel):
    m = load(mech)
    chem = capi.FiniteChem(mech, "fp64")
    n = 3001  # ragged
    for call, seed in enumerate((31, 32)):
        sol, _ = states.chem_state(m, n, seed, fuel, grid=(n, 1, 1), progress="beta22", T_range=(300.0, 2400.0))
        rng = np.random.default_rng(seed)
        dts = torch.from_numpy(10 ** rng.uniform(-7, -5, n)).cuda()
        ref = torch.from_numpy(sol).cuda()
        got = ref.clone()
        st = chem.substep(ref, dts, P)
        failed = chem.substep_static(got, dts, P)
        torch.cuda.synchronize()
        assert failed == st["cells_failed"], call
        assert torch.equal(got, ref), call


def test_static_scratch_rejects_oversized_batch():
    chem = capi.FiniteChem("hydrogen", "fp64")
    nv = chem.nspecies + 1
    x = torch.zeros((nv, (1 << 18) + 1), dtype=torch.float64, device="cuda")
    with pytest.raises(capi.ChemError, match="static limit"):
        chem.substep_static(x, 1e-6, P)


def _cells(m, fuel, n, seed):
    sol, _ = states.chem_state(m, n, seed, fuel, grid=(n, 1, 1), progress="beta22", T_range=(300.0, 2400.0))
    return torch.from_numpy(sol).cuda()


def test_static_scratch_alternating_mechanisms_padded_and_scalar_dt():
    """Hydrogen and GRI-Mech handles alternate on the shared scratch (each call selects its
    mechanism's tables, nothing is re-copied), once with a padded leading dimension and once
    with a scalar dt; every result equals tng_substep_batch's on the same cells."""
    cases = [("hydrogen", "H2", 0), ("grimech30", "CH4", 1), ("hydrogen", "H2", 2), ("grimech30", "CH4", 3)]
    chems = {mech: capi.FiniteChem(mech, "fp64") for mech in ("hydrogen", "grimech30")}
    n, pad = 777, 41
    for mech, fuel, i in cases:
        chem = chems[mech]
        x = _cells(load(mech), fuel, n, 40 + i)
        if i % 2:  # padded: ld = n + pad
            wide = torch.full((x.shape[0], n + pad), float("nan"), dtype=torch.float64, device="cuda")
            wide[:, :n] = x
            got = wide[:, :n]
        else:
            got = x.clone()
        dt = 2e-6 if i >= 2 else torch.from_numpy(10 ** np.random.default_rng(i).uniform(-7, -5, n)).cuda()
        ref = x.clone()
        st = chem.substep(ref, dt, P)
        failed = chem.substep_static(got, dt, P)
        torch.cuda.synchronize()
        assert failed == st["cells_failed"], (mech, i)
        assert torch.equal(got, ref), (mech, i)
        if i % 2:
            assert torch.isnan(wide[:, n:]).all(), "cells past ncells were written"
