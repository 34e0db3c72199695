"""The Fortran-signature shims tng_prodrates_ / tng_compthermodata_ (PRODRATES, COMPTHERMODATA,
e.g. combustion/HYDROGENF.f90:4-277, :514-673) on the GPU against the CPU oracle, one cell per call
as finitechem_compute_rhs calls them. CDOT within 1e-10 of the cancellation-free scale
sum_r |nu_kr W_r|; slot rates within 1e-10 relative; h and cp within 1e-13 relative, on both sides
of the strict T > 1000 K switch."""
import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mech", ["hydrogen", "grimech30", "dme39"])
def test_shims_match_oracle(mech):
    from tiger_nga_b200 import capi
    from tiger_nga_b200.mechanism import load

    chem = capi.FiniteChem(mech, "fp64")
    o = Oracle(mech)
    nu = np.abs(load(mech).nu)
    rng = np.random.default_rng(3)
    for T in (300.0, 1000.0, np.nextafter(1000.0, 2000.0), 1850.0, 2900.0):
        C = 10.0 ** rng.uniform(-12, -2, chem.nspecies)
        P = 101325.0 * rng.uniform(0.5, 4.0)
        cdot, w = chem.prodrates_cell(C, T, P)
        cd_ref, w_ref, _, _ = o.prodrates(C, T, P)
        scale = nu @ np.abs(w_ref) + 1e-300
        assert np.max(np.abs(cdot - cd_ref) / scale) <= 1e-10
        assert np.max(np.abs(w - w_ref) / np.maximum(np.abs(w_ref), 1e-300)) <= 1e-10
        hk, cp = chem.thermo_cell(T)
        h_ref, cp_ref = o.thermo(T)
        assert np.max(np.abs(hk - h_ref) / np.maximum(np.abs(h_ref), 1.0)) <= 1e-13
        assert np.max(np.abs(cp - cp_ref) / cp_ref) <= 1e-13
    chem.close()
