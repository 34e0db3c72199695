"""The drop-in for finitechem_source_chemistry(RHO_, SC_): the host solver's own Fortran-ordered
arrays with ghost layers, a mask, extra scalars around the species block -- against the batch
substep on the same interior cells and the reference's HR / chemsrc formulas
(combustion/finitechem.f90:1002-1057)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tiger_nga_b200 import capi, states  # noqa: E402
from tiger_nga_b200.mechanism import load  # noqa: E402

pytestmark = pytest.mark.gpu
P = 101325.0


def test_source_chemistry_matches_batch_and_reference_formulas():
    mech = "grimech30"
    m = load(mech)
    ns = m.ns
    g = 2
    nx, ny, nz = 6, 5, 4
    imin, jmin, kmin = 1, 1, 1
    imino, jmino, kmino = imin - g, jmin - g, kmin - g
    nxo, nyo, nzo = nx + 2 * g, ny + 2 * g, nz + 2 * g
    isc_sc, isc_T = 3, 3 + ns  # two other scalars (e.g. velocity-like) before the species, T after
    nscalar = isc_T + 1
    n_all = nxo * nyo * nzo
    sol, info = states.chem_state(m, n_all, 21, "CH4", grid=(n_all, 1, 1))
    Y = info["Y"].T.reshape(nxo, nyo, nzo, ns, order="F")
    T = info["T"].reshape(nxo, nyo, nzo, order="F")
    RHO = np.asfortranarray(info["rho"].reshape(nxo, nyo, nzo, order="F"))
    SC = np.zeros((nxo, nyo, nzo, nscalar), order="F")
    SC[..., 0] = 7.0
    SC[..., 1] = -3.0
    SC[..., isc_sc - 1:isc_sc - 1 + ns] = Y
    SC[..., isc_T - 1] = T
    SC[..., nscalar - 1] = 42.0
    mask = np.zeros((nxo, nyo), dtype=np.int32, order="F")
    mask[g + 1, g + 2] = 1  # a wall column
    HR = np.full((nxo, nyo, nzo), 3.0, order="F")
    CS = np.full((nxo, nyo, nzo, 3), 1e-60, order="F")
    names = m.species
    ext = dict(imino=imino, imaxo=imino + nxo - 1, jmino=jmino, jmaxo=jmino + nyo - 1, kmino=kmino,
               kmaxo=kmino + nzo - 1, imin=imin, imax=imin + nx - 1, jmin=jmin, jmax=jmin + ny - 1, kmin=kmin,
               kmax=kmin + nz - 1, nscalar=nscalar, isc_sc=isc_sc, isc_T=isc_T,
               isc_H2O=isc_sc + names.index("H2O"), isc_CO=isc_sc + names.index("CO"),
               isc_CO2=isc_sc + names.index("CO2"))
    SC0 = SC.copy()
    dt = 1e-6
    chem = capi.FiniteChem(mech, "fp64")
    chem.source_chemistry(RHO, SC, ext, dt, P, mask=mask, HR=HR, chemsrc=CS)
    # the same interior cells through the batch substep
    sl = (slice(g, g + nx), slice(g, g + ny), slice(g, g + nz))
    r = RHO[sl].reshape(-1, order="F")
    state = np.empty((ns + 1, r.size))
    state[:ns] = np.maximum(r[None, :] * SC0[sl + (slice(isc_sc - 1, isc_sc - 1 + ns),)].reshape(-1, ns, order="F").T, 0)
    state[ns] = r * SC0[sl + (isc_T - 1,)].reshape(-1, order="F")
    old = state.copy()
    masked = np.zeros((nx, ny, nz), bool)
    masked[1, 2, :] = True
    dts = np.where(masked.reshape(-1, order="F"), 0.0, dt)
    chem.substep(state, dts, P)
    Yn = (state[:ns] / r[None, :]).T.reshape(nx, ny, nz, ns, order="F")
    Tn = (state[ns] / r).reshape(nx, ny, nz, order="F")
    got_Y = SC[sl + (slice(isc_sc - 1, isc_sc - 1 + ns),)]
    got_T = SC[sl + (isc_T - 1,)]
    assert np.array_equal(got_Y[~masked], Yn[~masked])
    assert np.array_equal(got_T[~masked], Tn[~masked])
    # masked cells, ghost layers and the other scalars untouched
    assert np.array_equal(SC[g + 1, g + 2, g:g + nz], SC0[g + 1, g + 2, g:g + nz])
    ghost = np.ones((nxo, nyo, nzo), bool)
    ghost[sl] = False
    assert np.array_equal(SC[ghost], SC0[ghost])
    for q in (0, 1, nscalar - 1):
        assert np.array_equal(SC[..., q], SC0[..., q])
    # HR = Cp(new Y, new T) * d(rho T)/dt and chemsrc = d(rho Y)/dt (finitechem.f90:1047-1057)
    tab = np.where((Tn > m.tmid)[..., None, None], m.th_hi[None, None, None], m.th_lo[None, None, None])
    t = Tn[..., None]
    cp = tab[..., 0] * (tab[..., 7] + t * (tab[..., 8] + t * (tab[..., 9] + t * (tab[..., 10] + t * tab[..., 11]))))
    cpm = np.sum(Yn * cp, axis=-1)
    dT = ((state[ns] - old[ns]) / dt).reshape(nx, ny, nz, order="F")
    hr = HR[sl]
    assert np.allclose(hr[~masked], (cpm * dT)[~masked], rtol=1e-12, atol=0)
    assert np.all(hr[masked] == 3.0)
    for q, nm in enumerate(("H2O", "CO", "CO2")):
        k = names.index(nm)
        ref = ((state[k] - old[k]) / dt).reshape(nx, ny, nz, order="F")
        assert np.allclose(CS[sl + (q,)][~masked], ref[~masked], rtol=1e-12, atol=1e-300)
