"""Seeded synthetic chemistry states (the reference ships no input decks or datasets).

The recipe follows the reference's own finite-chemistry initial-condition tool
(tools/init_flow/ignition.f90:156-501): mix a fuel stream and an air stream by a mixture
fraction Z (ignition.f90:350-472), blend toward complete-combustion products, clip,
renormalise and form the ideal-gas density rho = P W_mix / (R T). Air is O2 + 3.76 N2 by mole
(ignition.f90:178), R = 8314.34 (ignition.f90:171).

* Z is a smooth seeded field: the sum of 16 Fourier modes with random integer wave-vectors
  (|k| <= 4), phases U[0, 2pi) and amplitudes N(0, 1), min-max mapped to [0, 1].
* Progress c in [0, 1] blends the unburnt mixture (Y_u, T_u) with complete-combustion products
  (Y_b, T_ad), T_ad from the enthalpy balance h(Y_b, T_ad) = h(Y_u, T_u) with the mechanism's
  own NASA polynomials.
* Minor species are set log-uniform in a range, then Y is renormalised to sum to 1.

States are returned species-major: ``sol[v, i]`` with ``v = 0..N-1`` the partial densities
rho*Y_k and ``v = N`` rho*T -- the CVODE state vector of finitechem.f90:1002-1003.
"""
from __future__ import annotations

import numpy as np

from .mechanism import Mechanism

R_CST = 8314.34
P_ATM = 101325.0


def fourier_field(shape, seed: int, modes: int = 16, kmax: int = 4) -> np.ndarray:
    """Smooth periodic field on a grid, min-max mapped to [0, 1]; float64, C order."""
    rng = np.random.default_rng(seed)
    ks = []
    while len(ks) < modes:
        k = rng.integers(-kmax, kmax + 1, size=3)
        if 0 < np.sqrt((k * k).sum()) <= kmax:
            ks.append(k)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    amp = rng.normal(size=modes)
    axes = [np.arange(n, dtype=np.float64) / n for n in shape]
    f = np.zeros(shape)
    for k, ph, a in zip(ks, phase, amp):
        # separable phase: cos(2pi(k.x) + ph)
        arg = (2 * np.pi * k[0] * axes[0])[:, None, None] + (2 * np.pi * k[1] * axes[1])[None, :, None] \
            + (2 * np.pi * k[2] * axes[2])[None, None, :]
        f += a * np.cos(arg + ph)
    lo, hi = f.min(), f.max()
    if not hi > lo:
        return np.full(shape, 0.5)
    return (f - lo) / (hi - lo)


def thermo_h(mech: Mechanism, T: np.ndarray) -> np.ndarray:
    """Species enthalpies h_k(T) [J/kg], shape (N, len(T)) (COMPTHERMODATA)."""
    T = np.atleast_1d(T).astype(np.float64)
    out = np.empty((mech.ns, T.size))
    for tab, mask in ((mech.th_hi, T > mech.tmid), (mech.th_lo, ~(T > mech.tmid))):
        t = T[mask]
        c = tab
        poly = c[:, 1, None] + t * (c[:, 2, None] + t * (c[:, 3, None] + t * (c[:, 4, None] + t * c[:, 5, None])))
        out[:, mask] = c[:, 0, None] * (t * poly + c[:, 6, None])
    return out


def thermo_cp(mech: Mechanism, T: np.ndarray) -> np.ndarray:
    T = np.atleast_1d(T).astype(np.float64)
    out = np.empty((mech.ns, T.size))
    for tab, mask in ((mech.th_hi, T > mech.tmid), (mech.th_lo, ~(T > mech.tmid))):
        t = T[mask]
        c = tab
        out[:, mask] = c[:, 0, None] * (c[:, 7, None] + t * (c[:, 8, None] + t * (c[:, 9, None] + t * (
            c[:, 10, None] + t * c[:, 11, None]))))
    return out


def _idx(mech: Mechanism, name: str) -> int:
    return mech.species.index(name)


def streams(mech: Mechanism, fuel: str):
    """Mass fractions of the fuel and air streams."""
    W = mech.wmol
    yf = np.zeros(mech.ns)
    yf[_idx(mech, fuel)] = 1.0
    ya = np.zeros(mech.ns)
    xo2, xn2 = 1.0, 3.76
    mo2, mn2 = xo2 * W[_idx(mech, "O2")], xn2 * W[_idx(mech, "N2")]
    ya[_idx(mech, "O2")] = mo2 / (mo2 + mn2)
    ya[_idx(mech, "N2")] = mn2 / (mo2 + mn2)
    return yf, ya


def burnt(mech: Mechanism, fuel: str, Yu: np.ndarray) -> np.ndarray:
    """Complete combustion of a fuel/air mixture (Burke-Schumann products), Yu shape (N, n)."""
    W = mech.wmol
    comp = dict(zip(mech.elements, mech.elem[:, _idx(mech, fuel)]))
    nc, nh, no = comp.get("C", 0.0), comp.get("H", 0.0), comp.get("O", 0.0)
    o2_per_fuel = nc + nh / 4.0 - no / 2.0
    f, o2 = _idx(mech, fuel), _idx(mech, "O2")
    nf = Yu[f] / W[f]
    no2 = Yu[o2] / W[o2]
    burn = np.minimum(nf, no2 / o2_per_fuel)
    Yb = Yu.copy()
    Yb[f] -= burn * W[f]
    Yb[o2] -= burn * o2_per_fuel * W[o2]
    if nc > 0:
        Yb[_idx(mech, "CO2")] += burn * nc * W[_idx(mech, "CO2")]
    Yb[_idx(mech, "H2O")] += burn * nh / 2.0 * W[_idx(mech, "H2O")]
    return np.maximum(Yb, 0.0)


def adiabatic_T(mech: Mechanism, Yu, Tu, Yb, iters: int = 40) -> np.ndarray:
    """T_ad with sum_k Yb_k h_k(T_ad) = sum_k Yu_k h_k(Tu) (Newton on the NASA polynomials)."""
    hu = np.einsum("kn,kn->n", Yu, thermo_h(mech, Tu))
    T = np.full(hu.shape, 2000.0)
    for _ in range(iters):
        hb = np.einsum("kn,kn->n", Yb, thermo_h(mech, T))
        cp = np.einsum("kn,kn->n", Yb, thermo_cp(mech, T))
        T = np.clip(T - (hb - hu) / cp, 250.0, 4500.0)
    return T


def chem_state(mech: Mechanism, ncells: int, seed: int, fuel: str, T_fuel: float = 300.0, T_air: float = 300.0,
               minor=(1e-10, 1e-3), minor_species=None, progress: str = "uniform", T_range=None,
               grid=None, p: float = P_ATM, z=None, c=None):
    """Seeded state batch. Returns (sol (N+1, ncells), info dict with Y, T, rho, Z, c).

    progress: 'uniform' (c ~ U[0,1]) or 'beta22' (c ~ Beta(2,2)); with T_range=(lo, hi) the
    temperature is lo + c (hi - lo) instead of the burnt/unburnt blend. z and c, when given,
    are the mixture fraction and progress of every cell.
    """
    rng = np.random.default_rng(seed + 7919)
    if z is None:
        if grid is None:
            side = int(round(ncells ** (1.0 / 3.0)))
            grid = (side, side, side) if side ** 3 == ncells else (ncells, 1, 1)
        z = fourier_field(grid, seed).reshape(-1)[:ncells]
    Z = np.asarray(z, dtype=np.float64).reshape(-1)
    yf, ya = streams(mech, fuel)
    Yu = yf[:, None] * Z[None, :] + ya[:, None] * (1.0 - Z[None, :])
    Tu = T_fuel * Z + T_air * (1.0 - Z)
    Yb = burnt(mech, fuel, Yu)
    # T_ad depends on Z only: solve the enthalpy balance on a Z table and interpolate
    zt = np.linspace(0.0, 1.0, 2049)
    Yut = yf[:, None] * zt[None, :] + ya[:, None] * (1.0 - zt[None, :])
    Tbt = adiabatic_T(mech, Yut, T_fuel * zt + T_air * (1.0 - zt), burnt(mech, fuel, Yut))
    Tb = np.interp(Z, zt, Tbt)
    if c is not None:
        c = np.asarray(c, dtype=np.float64).reshape(-1)
    elif progress == "uniform":
        c = rng.uniform(0.0, 1.0, ncells)
    elif progress == "beta22":
        c = rng.beta(2.0, 2.0, ncells)
    else:
        raise ValueError(progress)
    Y = (1.0 - c)[None, :] * Yu + c[None, :] * Yb
    if T_range is None:
        T = (1.0 - c) * Tu + c * Tb
    else:
        T = T_range[0] + c * (T_range[1] - T_range[0])
    majors = {fuel, "O2", "N2", "H2O", "CO2"}
    if minor_species is None:
        minor_species = [s for s in mech.species if s not in majors and s != "AR"]
    lo, hi = np.log10(minor[0]), np.log10(minor[1])
    for s in minor_species:
        Y[_idx(mech, s)] = 10.0 ** rng.uniform(lo, hi, ncells)
    Y = np.clip(Y, 0.0, 1.0)
    Y /= Y.sum(axis=0, keepdims=True)
    wmix = 1.0 / (Y / mech.wmol[:, None]).sum(axis=0)
    rho = p * wmix / (R_CST * T)
    sol = np.empty((mech.ns + 1, ncells))
    sol[:mech.ns] = rho[None, :] * Y
    sol[mech.ns] = rho * T
    return sol, {"Y": Y, "T": T, "rho": rho, "Z": Z, "c": c, "p": p}


# ---- the workloads, by what they are -------------------------------------------------------

def h2_cube(mech: Mechanism, n: int = 32, seed: int = 20261203):
    """H2/air, n^3 cells, radicals H, O, OH, HO2, H2O2 log-uniform in [1e-8, 1e-3]."""
    return chem_state(mech, n ** 3, seed, "H2", minor=(1e-8, 1e-3),
                      minor_species=["H", "O", "OH", "HO2", "H2O2"], grid=(n, n, n))


def ch4_cube(mech: Mechanism, n: int = 128, seed: int = 20261204, progress: str = "uniform", T_range=None):
    """CH4/air, n^3 cells, minor species log-uniform in [1e-10, 1e-3]."""
    return chem_state(mech, n ** 3, seed, "CH4", minor=(1e-10, 1e-3), grid=(n, n, n), progress=progress,
                      T_range=T_range)


def mixing_layer(mech: Mechanism, shape=(256, 192, 192), seed: int = 20261205, fuel: str = "CH3OCH3",
                 T_fuel: float = 400.0, T_air: float = 300.0, thickness: float = 0.08, amp: float = 0.1,
                 minor=(1e-10, 1e-3), p: float = P_ATM, chunk: int = 1 << 20):
    """Temporal mixing layer on a (nx, ny, nz) grid: fuel above air along y.

    Z = (1 + tanh((y - 1/2) / thickness)) / 2 + amp * (2 F - 1), clipped to [0, 1], with F a seeded
    smooth Fourier field in [0, 1]; the burning fraction c is a second seeded smooth field, which
    blends the unburnt mixture with its complete-combustion products (T up to adiabatic); minor
    species log-uniform in ``minor``. Built in chunks of cells (memory bounded). Returns
    (sol (N+1, ncells) C-ordered over (x, y, z), info with Z and c).
    """
    nx, ny, nz = shape
    y = (np.arange(ny, dtype=np.float64) + 0.5) / ny
    prof = 0.5 * (1.0 + np.tanh((y - 0.5) / thickness))
    Z = np.clip(prof[None, :, None] + amp * (2.0 * fourier_field(shape, seed) - 1.0), 0.0, 1.0).reshape(-1)
    c = fourier_field(shape, seed + 1).reshape(-1)
    n = Z.size
    sol = np.empty((mech.ns + 1, n))
    for k, lo in enumerate(range(0, n, chunk)):
        hi = min(n, lo + chunk)
        part, _ = chem_state(mech, hi - lo, seed + 101 * (k + 1), fuel, T_fuel=T_fuel, T_air=T_air, minor=minor,
                             p=p, z=Z[lo:hi], c=c[lo:hi])
        sol[:, lo:hi] = part
    return sol, {"Z": Z, "c": c, "shape": shape}
