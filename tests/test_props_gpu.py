"""Mixture properties on the GPU (tng_chem_density, tng_chem_transport) against the CPU oracle's
restatement of finitechem_W / _density / _viscosity / _diffusivity (combustion/finitechem.f90:
65-74, :324-487). FP64 bar: every output within 1e-10 relative of the oracle (the kernel
factors Wilke's pair sum into three dot products and folds W_mix out; the oracle keeps the
reference's pow-based order)."""
import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10


def cells(ns, n, seed):
    rng = np.random.default_rng(seed)
    Y = rng.dirichlet(np.full(ns, 0.25), n).T.copy()
    Y[:, : n // 50] *= rng.uniform(0, 1, (ns, n // 50)) ** 8  # traces
    Y[rng.integers(0, ns, n // 20), rng.integers(0, n, n // 20)] = -1e-12  # slightly negative entries
    Y[:, 1] = 0.0
    Y[0, 1] = 1.0  # pure first species
    Y[:, 2] *= 1.4  # sum above one
    T = rng.uniform(250.0, 3300.0, n)
    T[3], T[4], T[5] = 1000.0, 30.0, 5600.0  # NASA switch, both clips
    return Y, T


def rel_close(got, want, tol=TOL):
    got, want = np.asarray(got), np.asarray(want)
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    g, w = got[~nan], want[~nan]
    err = np.abs(g - w) / np.maximum(np.abs(w), 1e-300)
    assert err.max(initial=0.0) <= tol, float(err.max())
    return float(err.max(initial=0.0))


@pytest.mark.parametrize("mech", ["hydrogen", "grimech30", "dme39"])
@pytest.mark.parametrize("lm", ["ref", "f64"])
def test_batch_properties_match_oracle(mech, lm):
    import torch

    from tiger_nga_b200 import capi

    chem = capi.FiniteChem(mech, "fp64", literal_mode=lm)
    o = Oracle(mech, "f32" if lm == "ref" else "f64")
    ns = chem.nspecies
    n = 20011  # ragged against the 64-thread blocks
    Y, T = cells(ns, n, 7)
    lew = np.random.default_rng(8).uniform(0.6, 1.8, ns)
    sc = torch.from_numpy(np.vstack([Y, T[None]])).cuda()
    out = chem.mixture_props(sc, p_thermo=2.5e5, visc=True, diff=True, lewis=lew)
    torch.cuda.synchronize()
    want = o.props_batch(Y, T, p_thermo=2.5e5, lewis=lew)
    for k in ("wmix", "rho", "visc", "diff"):
        rel_close(out[k].cpu().numpy(), want[k])
    chem.close()


def test_all_zero_cell_follows_the_reference():
    """A cell with no species: W_mix = 0/0 (NaN) and so rho and lambda/Cp are NaN, while the
    viscosity sum skips every non-positive species and stays 0 -- as in the reference."""
    import torch

    from tiger_nga_b200 import capi

    chem = capi.FiniteChem("hydrogen", "fp64")
    o = Oracle("hydrogen")
    Y = np.zeros((chem.nspecies, 3))
    Y[2, 1] = 1.0
    Y[:, 2] = 1.0 / chem.nspecies
    T = np.array([800.0, 800.0, 1500.0])
    sc = torch.from_numpy(np.vstack([Y, T[None]])).cuda()
    out = chem.mixture_props(sc, p_thermo=101325.0, visc=True, diff=True)
    torch.cuda.synchronize()
    want = o.props_batch(Y, T, p_thermo=101325.0)
    assert np.isnan(want["rho"][0]) and want["visc"][0] == 0.0
    for k in want:
        rel_close(out[k].cpu().numpy(), want[k])
    chem.close()


def test_visc_alone_diff_alone_and_fused_agree():
    import torch

    from tiger_nga_b200 import capi

    chem = capi.FiniteChem("grimech30", "fp64")
    Y, T = cells(chem.nspecies, 4096, 9)
    sc = torch.from_numpy(np.vstack([Y, T[None]])).cuda()
    both = chem.mixture_props(sc, visc=True, diff=True)
    v = chem.mixture_props(sc, visc=True)
    d = chem.mixture_props(sc, diff=True)
    torch.cuda.synchronize()
    rel_close(v["visc"].cpu().numpy(), both["visc"].cpu().numpy(), 1e-14)
    rel_close(d["diff"].cpu().numpy(), both["diff"].cpu().numpy(), 1e-14)
    chem.close()


def _block(mech, seed):
    """A padded Fortran block (ghosts, extra scalars, a mask) as the host solver holds it."""
    o = Oracle(mech)
    ns = o.ns
    imino, imaxo, jmino, jmaxo, kmino, kmaxo = -2, 9, -1, 5, 0, 4
    nxo, nyo, nzo = imaxo - imino + 1, jmaxo - jmino + 1, kmaxo - kmino + 1
    nscalar = ns + 3  # ZMIX, species, T, one more scalar
    isc_zmix, isc_sc, isc_T = 1, 2, ns + 2
    vol = nxo * nyo * nzo
    Y, T = cells(ns, vol, seed)
    SC = np.zeros((nxo, nyo, nzo, nscalar), order="F")
    SC[..., isc_sc - 1:isc_sc - 1 + ns] = Y.T.reshape(nzo, nyo, nxo, ns).transpose(2, 1, 0, 3)
    SC[..., isc_T - 1] = T.reshape(nzo, nyo, nxo).transpose(2, 1, 0)
    SC[..., 0] = 0.3
    SC[..., ns + 2] = 7.0
    mask = np.zeros((nxo, nyo), dtype=np.int32, order="F")
    mask[2:4, 1] = 1
    mask[0, :] = 2  # only mask == 1 is skipped
    ext = dict(imino=imino, imaxo=imaxo, jmino=jmino, jmaxo=jmaxo, kmino=kmino, kmaxo=kmaxo, imin=imino + 2,
               imax=imaxo - 2, jmin=jmino + 1, jmax=jmaxo - 1, kmin=kmino, kmax=kmaxo, nscalar=nscalar,
               isc_sc=isc_sc, isc_T=isc_T, isc_H2O=0, isc_CO=0, isc_CO2=0)
    return o, SC, mask, ext, (nxo, nyo, nzo), isc_zmix


@pytest.mark.parametrize("mech", ["hydrogen", "grimech30"])
def test_fortran_drop_ins_on_padded_block(mech):
    from tiger_nga_b200 import capi

    chem = capi.FiniteChem(mech, "fp64")
    o, SC, mask, ext, (nxo, nyo, nzo), isc_zmix = _block(mech, 3)
    ns = o.ns
    lew = np.linspace(0.8, 1.3, ns)
    RHO = np.full((nxo, nyo, nzo), -1.0, order="F")
    W = np.full((nxo, nyo, nzo), -2.0, order="F")
    VISC = np.full((nxo, nyo, nzo), -3.0, order="F")
    DIFF = np.full(SC.shape, -4.0, order="F")
    SC0 = SC.copy(order="F")
    chem.density(RHO, SC, ext, 1.2e5, mask=mask, W=W)
    chem.transport(SC, ext, VISC=VISC, DIFF=DIFF, mask=mask, lewis=lew, isc_zmix=isc_zmix)
    assert np.array_equal(SC, SC0)
    # expected: every cell of the padded block, in Fortran order, through the oracle
    Yf = SC[..., 1:1 + ns].reshape(-1, ns, order="F").T.copy()
    Tf = SC[..., ns + 1].reshape(-1, order="F").copy()
    want = o.props_batch(Yf, Tf, p_thermo=1.2e5, lewis=lew)
    live = (np.broadcast_to(mask[:, :, None], (nxo, nyo, nzo)) != 1).reshape(-1, order="F")
    assert 0 < live.sum() < live.size
    flat = lambda a: a.reshape(-1, order="F")  # noqa: E731
    rel_close(flat(RHO)[live], want["rho"][live])
    rel_close(flat(W)[live], want["wmix"][live])
    rel_close(flat(VISC)[live], want["visc"][live])
    D = DIFF.reshape(-1, SC.shape[3], order="F")
    rel_close(D[live, 1:1 + ns].T, want["diff"][:ns, live])
    rel_close(D[live, ns + 1], want["diff"][ns, live])
    rel_close(D[live, isc_zmix - 1], want["diff"][ns, live])
    # masked cells and the other scalar column are untouched
    assert (flat(RHO)[~live] == -1.0).all() and (flat(W)[~live] == -2.0).all() and (flat(VISC)[~live] == -3.0).all()
    assert (D[~live] == -4.0).all() and (D[:, ns + 2] == -4.0).all()
    chem.close()


def test_argument_errors():
    from tiger_nga_b200 import capi

    chem = capi.FiniteChem("hydrogen", "fp64")
    o, SC, mask, ext, (nxo, nyo, nzo), isc_zmix = _block("hydrogen", 4)
    VISC = np.zeros((nxo, nyo, nzo), order="F")
    DIFF = np.zeros(SC.shape, order="F")
    with pytest.raises(capi.ChemError):
        chem.transport(SC, ext, VISC=VISC, DIFF=DIFF, isc_zmix=ext["isc_sc"])  # ZMIX inside the species block
    with pytest.raises(capi.ChemError):
        chem.transport(SC, ext, VISC=VISC, lewis=np.zeros(o.ns))
    with pytest.raises(capi.ChemError):
        chem.density(VISC, SC, ext, -1.0)
    bad = dict(ext, isc_T=ext["isc_sc"])
    with pytest.raises(capi.ChemError):
        chem.density(VISC, SC, bad, 1e5)
    chem.close()
