"""Python side of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this
module, and only as the checker or the timed CPU baseline. The product never imports it.

* :class:`Oracle` loads a mechanism table (the JSON under ``tiger_nga_b200/mechanisms``),
  turns every literal into the double the reference binary would use (default-real literals
  rounded to float32, Makefile.in:23-24), and drives ``chem_oracle.c`` -- the table-driven
  restatement of PRODRATES / GETLINDRATECOEFF / COMPTHERMODATA / finitechem_compute_rhs, and
  ``props_oracle.c`` for the mixture properties (finitechem_W / _density / _viscosity /
  _diffusivity).
* :class:`Reference` drives ``oracle/_ref/libref_mech.so``, the reference's own Fortran
  mechanism routines transliterated statement by statement to C by ``oracle/f90_to_c.py``.
  It exists only where that library was built (it needs the reference tree to build).

The literal-kind rule and table flattening are written here independently of the product's
loader on purpose.
"""
from __future__ import annotations

import ctypes
import json
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
MECH_DIR = os.path.join(REPO, "tiger_nga_b200", "mechanisms")
LIB = os.path.join(HERE, "_build", "libchem_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_mech.so")
REF_FILEIO = os.path.join(HERE, "_ref", "libref_fileio.so")


def build_oracle(force: bool = False) -> str:
    """Compile chem_oracle.c (and solver_oracle.c when present) with gcc + OpenMP."""
    srcs = [os.path.join(HERE, f) for f in ("chem_oracle.c", "solver_oracle.c", "props_oracle.c")
            if os.path.exists(os.path.join(HERE, f))]
    newest = max(os.path.getmtime(s) for s in srcs + [os.path.join(HERE, "orc_mech.h")])
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        tmp = LIB + f".{os.getpid()}.tmp"
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
                               "-o", tmp] + srcs + ["-lm"])
        os.replace(tmp, LIB)
    return LIB


def _lit(text, mode="f32"):
    t = text.strip()
    neg = t.startswith("-")
    body = t[1:] if neg else t
    if body.upper().endswith("_DP"):
        v = float(body[:-3].replace("D", "E").replace("d", "e"))
    elif "d" in body.lower():
        v = float(body.replace("D", "E").replace("d", "e"))
    elif "." in body or "e" in body.lower():
        v = float(body)
        if mode == "f32":
            v = struct.unpack("<f", struct.pack("<f", v))[0]
    else:
        v = float(int(body))
    return -v if neg else v


class _Mech(ctypes.Structure):
    _fields_ = [
        ("ns", ctypes.c_int), ("nslot", ctypes.c_int), ("nm", ctypes.c_int), ("nfo", ctypes.c_int),
        ("rgas", ctypes.c_double), ("troe", ctypes.c_double * 7),
        ("tb_ptr", ctypes.c_void_p), ("tb_sp", ctypes.c_void_p), ("tb_coef", ctypes.c_void_p),
        ("k_flags", ctypes.c_void_p), ("kA", ctypes.c_void_p), ("kn", ctypes.c_void_p), ("kE", ctypes.c_void_p),
        ("k_fo", ctypes.c_void_p),
        ("f0_flags", ctypes.c_void_p), ("fi_flags", ctypes.c_void_p),
        ("f0A", ctypes.c_void_p), ("f0n", ctypes.c_void_p), ("f0E", ctypes.c_void_p),
        ("fiA", ctypes.c_void_p), ("fin", ctypes.c_void_p), ("fiE", ctypes.c_void_p),
        ("fc_ptr", ctypes.c_void_p), ("fc_form", ctypes.c_void_p), ("fc_a", ctypes.c_void_p),
        ("fc_x", ctypes.c_void_p), ("fo_M", ctypes.c_void_p),
        ("w_ptr", ctypes.c_void_p), ("w_sp", ctypes.c_void_p), ("w_M", ctypes.c_void_p),
        ("cd_ptr", ctypes.c_void_p), ("cd_sign", ctypes.c_void_p), ("cd_slot", ctypes.c_void_p),
        ("cd_coef", ctypes.c_void_p),
        ("tmid", ctypes.c_double), ("th_hi", ctypes.c_void_p), ("th_lo", ctypes.c_void_p), ("wmol", ctypes.c_void_p),
        ("nu", ctypes.c_void_p), ("eff", ctypes.c_void_p),
    ]


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """Table-driven FP64 restatement of the reference chemistry, one mechanism."""

    def __init__(self, name: str, literal_mode: str = "f32"):
        self.name = name
        self.mode = literal_mode
        with open(os.path.join(MECH_DIR, name + ".json")) as fh:
            tab = json.load(fh)
        self.tab = tab
        L = lambda t: _lit(t, literal_mode)  # noqa: E731
        ns, nslot, nm = tab["n_species"], tab["n_slots"], tab["n_thirdbody"]
        self.ns, self.nslot, self.nm = ns, nslot, nm
        keep = []

        def I(x):  # noqa: E743
            a = np.ascontiguousarray(np.asarray(x, dtype=np.int32))
            keep.append(a)
            return a

        def D(x):
            a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
            keep.append(a)
            return a

        tb_ptr, tb_sp, tb_coef = [0], [], []
        for terms in tab["third_body"]:
            for s, c in terms:
                tb_sp.append(s)
                tb_coef.append(L(c))
            tb_ptr.append(len(tb_sp))

        def arr_flags(d):
            return (2 if d["n"] is not None else 0) | (4 if d["E"] is not None else 0)

        kfl, kA, kn, kE, kfo = [], [], [], [], []
        f0fl, fifl, f0A, f0n, f0E, fiA, fin, fiE, fcp, fcf, fca, fcx, foM = ([] for _ in range(13))
        fcp.append(0)
        for k in tab["k"]:
            if k["type"] == "falloff":
                kfl.append(1)
                kA.append(0.0), kn.append(0.0), kE.append(0.0)
                kfo.append(len(foM))
                for d, fl, A, n, E in ((k["k0"], f0fl, f0A, f0n, f0E), (k["kinf"], fifl, fiA, fin, fiE)):
                    fl.append(arr_flags(d))
                    A.append(L(d["A"]))
                    n.append(L(d["n"]) if d["n"] is not None else 0.0)
                    E.append(L(d["E"]) if d["E"] is not None else 0.0)
                for t in k["fc"]:
                    fcf.append(0 if t["form"] == "T_over" else 1)
                    fca.append(L(t["a"]))
                    fcx.append(L(t["x"]))
                fcp.append(len(fca))
                foM.append(k["M"])
            else:
                kfl.append(arr_flags(k))
                kA.append(L(k["A"]))
                kn.append(L(k["n"]) if k["n"] is not None else 0.0)
                kE.append(L(k["E"]) if k["E"] is not None else 0.0)
                kfo.append(-1)
        w_ptr, w_sp, w_M = [0], [], []
        for w in tab["w"]:
            w_sp += w["C"]
            w_ptr.append(len(w_sp))
            w_M.append(w["M"])
        cd_ptr, cd_sign, cd_slot, cd_coef = [0], [], [], []
        for terms in tab["cdot"]:
            for sgn, c, r in terms:
                cd_sign.append(sgn)
                cd_coef.append(L(c))
                cd_slot.append(r)
            cd_ptr.append(len(cd_slot))

        def thermo(rng):
            out = []
            for e in tab["thermo"][rng]:
                out += [L(e["c0"])] + [L(a) for a in e["a"]] + [L(e["a6"])] + [L(b) for b in e["b"]]
            return out

        self.wmol = D([L(x) for x in tab["molar_mass"]])
        self.mucoeff = D([L(x) for x in tab["mucoeff"]])
        self.koveps = D([L(x) for x in tab["koveps"]])
        nu = np.zeros((ns, nslot))
        for k, terms in enumerate(tab["cdot"]):
            for sgn, c, r in terms:
                nu[k, r] += sgn * L(c)
        eff = np.zeros((max(nm, 1), ns))
        for j, terms in enumerate(tab["third_body"]):
            for s_, c in terms:
                eff[j, s_] += L(c)
        self.nu_dense, self.eff_dense = D(nu), D(eff)
        m = _Mech()
        m.ns, m.nslot, m.nm, m.nfo = ns, nslot, nm, len(foM)
        m.rgas = L(tab["rgas"])
        m.troe[:] = [L("0.75"), L("1.27"), L("0.4"), L("0.67"), L("0.14"), L("1.0D-60"), L("1.0")]
        for fname, val in (("tb_ptr", I(tb_ptr)), ("tb_sp", I(tb_sp)), ("tb_coef", D(tb_coef)),
                           ("k_flags", I(kfl)), ("kA", D(kA)), ("kn", D(kn)), ("kE", D(kE)), ("k_fo", I(kfo)),
                           ("f0_flags", I(f0fl + [0])), ("fi_flags", I(fifl + [0])),
                           ("f0A", D(f0A + [0])), ("f0n", D(f0n + [0])), ("f0E", D(f0E + [0])),
                           ("fiA", D(fiA + [0])), ("fin", D(fin + [0])), ("fiE", D(fiE + [0])),
                           ("fc_ptr", I(fcp)), ("fc_form", I(fcf + [0])), ("fc_a", D(fca + [0])),
                           ("fc_x", D(fcx + [0])), ("fo_M", I(foM + [0])),
                           ("w_ptr", I(w_ptr)), ("w_sp", I(w_sp + [0])), ("w_M", I(w_M)),
                           ("cd_ptr", I(cd_ptr)), ("cd_sign", I(cd_sign + [0])), ("cd_slot", I(cd_slot + [0])),
                           ("cd_coef", D(cd_coef + [0])),
                           ("th_hi", D(thermo("hi"))), ("th_lo", D(thermo("lo"))), ("wmol", self.wmol),
                           ("nu", self.nu_dense), ("eff", self.eff_dense)):
            setattr(m, fname, _p(val))
        m.tmid = L(tab["thermo"]["tmid"])
        self._keep = keep
        self.m = m
        self.lib = ctypes.CDLL(build_oracle())
        self.lib.orc_prodrates.argtypes = [ctypes.POINTER(_Mech)] + [ctypes.c_void_p] * 5 + [ctypes.c_double] * 2
        self.lib.orc_thermo.argtypes = [ctypes.POINTER(_Mech), ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        self.lib.orc_rhs.argtypes = [ctypes.POINTER(_Mech), ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        self.lib.orc_rhs_batch.argtypes = [ctypes.POINTER(_Mech), ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                           ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        self.lib.orc_max_threads.restype = ctypes.c_int
        _solver_protos(self.lib)
        self.lib.orc_rhs_gross_batch.argtypes = [ctypes.POINTER(_Mech), ctypes.c_void_p, ctypes.c_double,
                                                 ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        self.lib.orc_rates_batch.argtypes = [ctypes.POINTER(_Mech), ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                             ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        self.lib.orc_props_batch.argtypes = ([ctypes.POINTER(_Mech)] + [ctypes.c_void_p] * 5 +
                                             [ctypes.c_int64, ctypes.c_int64, ctypes.c_double] +
                                             [ctypes.c_void_p] * 4 + [ctypes.c_int])

    # ---- single cell --------------------------------------------------------------------
    def prodrates(self, C, T, P):
        """(cdot, W, K, M) for concentrations C [kmol/m^3], T [K], P [Pa]."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        cd = np.zeros(self.ns)
        W = np.zeros(self.nslot)
        K = np.zeros(self.nslot)
        M = np.zeros(max(self.nm, 1))
        self.lib.orc_prodrates(ctypes.byref(self.m), _p(cd), _p(W), _p(K), _p(C), _p(M), float(T), float(P))
        return cd, W, K, M

    def thermo(self, T):
        h = np.zeros(self.ns)
        cp = np.zeros(self.ns)
        self.lib.orc_thermo(ctypes.byref(self.m), float(T), _p(h), _p(cp))
        return h, cp

    def rhs(self, sol, p):
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        out = np.zeros(self.ns + 1)
        self.lib.orc_rhs(ctypes.byref(self.m), _p(sol), float(p), _p(out))
        return out

    # ---- batch (species-major) ------------------------------------------------------------
    def rhs_batch(self, sol, p, nthreads=0):
        """sol: (N+1, ncells) float64 C-contiguous, species-major. Returns rhs of the same shape."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        out = np.empty_like(sol)
        self.lib.orc_rhs_batch(ctypes.byref(self.m), _p(sol), float(p), _p(out), sol.shape[1], sol.shape[1],
                               int(nthreads))
        return out

    def rhs_gross_batch(self, sol, p, nthreads=0):
        """Cancellation-free magnitude of each rhs entry (denominator of the normwise test)."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        out = np.empty_like(sol)
        self.lib.orc_rhs_gross_batch(ctypes.byref(self.m), _p(sol), float(p), _p(out), sol.shape[1], sol.shape[1],
                                     int(nthreads))
        return out

    def rates_batch(self, sol, p, nthreads=0):
        """Every slot's rate W_r, shape (nslot, ncells)."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        out = np.empty((self.nslot, sol.shape[1]))
        self.lib.orc_rates_batch(ctypes.byref(self.m), _p(sol), float(p), _p(out), sol.shape[1], sol.shape[1],
                                 sol.shape[1], int(nthreads))
        return out

    def props_batch(self, Y, T, p_thermo=101325.0, lewis=None, what=("wmix", "rho", "visc", "diff"), nthreads=0):
        """finitechem_W / _density / _viscosity / _diffusivity (finitechem.f90:65-74, :324-461) over a
        species-major batch: Y (N, ncells), T (ncells). Returns a dict of the requested outputs;
        'diff' is (N+1, ncells): lambda/Cp_mix/Lewis_k per species, then lambda/Cp_mix."""
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        n = Y.shape[1]
        out = {k: np.zeros((self.ns + 1, n) if k == "diff" else n) for k in what}
        lw = None if lewis is None else np.ascontiguousarray(lewis, dtype=np.float64)
        g = lambda k: _p(out[k]) if k in out else None  # noqa: E731
        self.lib.orc_props_batch(ctypes.byref(self.m), _p(self.mucoeff), _p(self.koveps),
                                 _p(lw) if lw is not None else None, _p(Y), _p(T), n, n, float(p_thermo),
                                 g("wmix"), g("rho"), g("visc"), g("diff"), int(nthreads))
        return out

    def max_threads(self):
        return self.lib.orc_max_threads()


class SolverCfg(ctypes.Structure):
    _fields_ = [("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("max_steps", ctypes.c_int),
                ("maxcor", ctypes.c_int), ("msbp", ctypes.c_int), ("dgmax", ctypes.c_double)]


class CellStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("nst", ctypes.c_int), ("nni", ctypes.c_int), ("nje", ctypes.c_int),
                ("nef", ctypes.c_int), ("ncf", ctypes.c_int), ("nrhs", ctypes.c_int), ("q", ctypes.c_int),
                ("h", ctypes.c_double)]


def _solver_protos(lib):
    lib.orc_jacobian.argtypes = [ctypes.POINTER(_Mech), ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                 ctypes.c_void_p]
    lib.orc_bdf_cell.argtypes = [ctypes.POINTER(_Mech), ctypes.POINTER(SolverCfg), ctypes.c_void_p, ctypes.c_double,
                                 ctypes.c_double, ctypes.POINTER(CellStats)]
    lib.orc_bdf_batch.argtypes = [ctypes.POINTER(_Mech), ctypes.POINTER(SolverCfg), ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_int64, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.orc_lu.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.orc_lu.restype = ctypes.c_int
    lib.orc_lu_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]


def solver_cfg(rtol=1e-6, atol=1e-12, max_steps=10000, maxcor=3, msbp=20, dgmax=0.3):
    return SolverCfg(rtol, atol, max_steps, maxcor, msbp, dgmax)


def _oracle_jacobian(self, u, p):
    u = np.ascontiguousarray(u, dtype=np.float64)
    f0 = self.rhs(u, p)
    J = np.zeros((self.ns + 1, self.ns + 1))
    self.lib.orc_jacobian(ctypes.byref(self.m), _p(u), float(p), _p(f0), _p(J))
    return J


def _oracle_substep_cell(self, u, dt, p, cfg=None):
    u = np.array(u, dtype=np.float64)
    st = CellStats()
    cfg = cfg or solver_cfg()
    self.lib.orc_bdf_cell(ctypes.byref(self.m), ctypes.byref(cfg), _p(u), float(dt), float(p), ctypes.byref(st))
    return u, {k: getattr(st, k) for k, _ in CellStats._fields_}


def _oracle_substep_batch(self, state, dt, p, cfg=None, nthreads=0):
    """Integrate a species-major batch (N+1, ncells) over dt (scalar or per cell)."""
    out = np.array(state, dtype=np.float64, order="C", copy=True)
    n = out.shape[1]
    cfg = cfg or solver_cfg()
    nst = np.zeros(n, dtype=np.int32)
    nni = np.zeros(n, dtype=np.int32)
    status = np.zeros(n, dtype=np.int32)
    if np.ndim(dt) == 0:
        dts, dts_p, dts_s = None, None, float(dt)
    else:
        dts = np.ascontiguousarray(dt, dtype=np.float64)
        dts_p, dts_s = _p(dts), 0.0
    self.lib.orc_bdf_batch(ctypes.byref(self.m), ctypes.byref(cfg), _p(out), n, n, dts_p, dts_s, float(p), _p(nst),
                           _p(nni), _p(status), int(nthreads))
    return out, {"nst": nst, "nni": nni, "status": status}


Oracle.jacobian = _oracle_jacobian
Oracle.substep_cell = _oracle_substep_cell
Oracle.substep_batch = _oracle_substep_batch


class Reference:
    """The reference's own mechanism routines, transliterated to C (oracle/_ref)."""

    def __init__(self, name: str):
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(REF_LIB)
        self.lib = ctypes.CDLL(REF_LIB)
        ns, nr, nm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        getattr(self.lib, f"ref_{name}_sizes")(ctypes.byref(ns), ctypes.byref(nr), ctypes.byref(nm))
        self.ns, self.nslot, self.nm = ns.value, nr.value, nm.value
        self._pr = getattr(self.lib, f"ref_{name}_prodrates")
        self._th = getattr(self.lib, f"ref_{name}_compthermodata")
        self._mm = getattr(self.lib, f"ref_{name}_getmolarmass")
        self._rb = getattr(self.lib, f"ref_{name}_rhs_batch")
        self._pb = getattr(self.lib, f"ref_{name}_props_batch", None)
        for f in (self._pr, self._th, self._mm, self._rb):
            f.restype = None
        mm = np.zeros(self.ns)
        self._mm(_p(mm))
        self.wmol = mm
        if self._pb is not None:
            self._pb.restype = None
            self._pb.argtypes = ([ctypes.c_void_p] * 2 + [ctypes.c_int64, ctypes.c_int64, ctypes.c_double] +
                                 [ctypes.c_void_p] * 5 + [ctypes.c_int])
            self.mucoeff, self.koveps = np.zeros(self.ns), np.zeros(self.ns)
            getattr(self.lib, f"ref_{name}_getmucoeff")(_p(self.mucoeff))
            getattr(self.lib, f"ref_{name}_getkovereps")(_p(self.koveps))

    def props_batch(self, Y, T, p_thermo=101325.0, lewis=None, what=("wmix", "rho", "visc", "diff"), nthreads=0):
        """The reference's finitechem_W / _density / _viscosity / _diffusivity over the
        transliterated getters; same outputs as :meth:`Oracle.props_batch`."""
        if self._pb is None:
            raise FileNotFoundError("oracle/_ref predates the property routines; rebuild it")
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        n = Y.shape[1]
        out = {k: np.zeros((self.ns + 1, n) if k == "diff" else n) for k in what}
        lw = None if lewis is None else np.ascontiguousarray(lewis, dtype=np.float64)
        g = lambda k: _p(out[k]) if k in out else None  # noqa: E731
        self._pb(_p(Y), _p(T), n, n, float(p_thermo), _p(lw) if lw is not None else None,
                 g("wmix"), g("rho"), g("visc"), g("diff"), int(nthreads))
        return out

    def rhs_batch(self, sol, p, nthreads=0):
        """finitechem_compute_rhs over a species-major batch, OpenMP over cells."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        out = np.empty_like(sol)
        f = self._rb
        f(_p(sol), ctypes.c_double(p), _p(out), ctypes.c_int64(sol.shape[1]), ctypes.c_int64(sol.shape[1]),
          ctypes.c_int(int(nthreads)))
        return out

    def prodrates(self, C, T, P):
        C = np.array(C, dtype=np.float64)
        cd, W, K, M = np.zeros(self.ns), np.zeros(self.nslot), np.zeros(self.nslot), np.zeros(self.nm)
        t, p = ctypes.c_double(T), ctypes.c_double(P)
        self._pr(_p(cd), _p(W), _p(K), _p(C), _p(M), ctypes.byref(t), ctypes.byref(p))
        return cd, W, K, M

    def thermo(self, T):
        h, cp = np.zeros(self.ns), np.zeros(self.ns)
        t = ctypes.c_double(T)
        self._th(_p(h), _p(cp), ctypes.byref(t))
        return h, cp

    def rhs(self, sol, p):
        """finitechem_compute_rhs (finitechem.f90:93-175) over the transliterated routines."""
        N = self.ns
        sol = np.asarray(sol, dtype=np.float64)
        rho = 0.0
        for k in range(N):
            rho = rho + sol[k]
        Y = sol[:N] / rho
        T = sol[N] / rho
        h, cp = self.thermo(T)
        cpmix = 0.0
        for k in range(N):
            cpmix = cpmix + Y[k] * cp[k]
        conc = sol[:N] / self.wmol
        cd, _, _, _ = self.prodrates(conc, T, p)
        out = np.zeros(N + 1)
        out[:N] = cd * self.wmol
        tmp = 0.0
        for k in range(N):
            tmp = tmp - h[k] * out[k]
        out[N] = tmp / cpmix
        return out


class RefFileIO:
    """The reference's own binary file library (library/fileio_c.c, built unchanged into
    oracle/_ref/libref_fileio.so), driven in the statement order of its data-file writer
    (tools/init_flow/param.f90:113-148, param_write_data) and reader (core/data.f90:217-284)."""

    def __init__(self):
        if not os.path.exists(REF_FILEIO):
            raise FileNotFoundError(REF_FILEIO)
        self.lib = ctypes.CDLL(REF_FILEIO)
        P = ctypes.POINTER(ctypes.c_int)
        self.lib.BINARY_FILE_OPEN.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, P, ctypes.c_int, ctypes.c_int]
        self.lib.BINARY_FILE_WRITE.argtypes = [P, ctypes.c_void_p, P, P, P]
        self.lib.BINARY_FILE_READ.argtypes = [P, ctypes.c_void_p, P, P, P]
        self.lib.BINARY_FILE_CLOSE.argtypes = [P, P]

    def _open(self, path, mode):
        unit, ierr = ctypes.c_int(), ctypes.c_int()
        p = path.encode()
        if len(p) >= 64:  # BINARY_FILE_OPEN copies the name into char[64] (library/fileio_c.c)
            raise ValueError(f"the reference's file library takes paths shorter than 64 bytes: {path}")
        self.lib.BINARY_FILE_OPEN(ctypes.byref(unit), p, mode.encode(), ctypes.byref(ierr), len(p), len(mode))
        if ierr.value:
            raise OSError(f"BINARY_FILE_OPEN failed on {path}")
        return unit

    def _io(self, f, unit, buf, count, size):
        c, s, e = ctypes.c_int(count), ctypes.c_int(size), ctypes.c_int()
        f(ctypes.byref(unit), buf, ctypes.byref(c), ctypes.byref(s), ctypes.byref(e))

    def write_data(self, path, data, names, dt=0.0, time=0.0):
        """param_write_data: data is (nx, ny, nz, nvar) in Fortran order, names up to 8 chars."""
        data = np.asfortranarray(data, dtype=np.float64)
        nx, ny, nz, nvar = data.shape
        u = self._open(path, "w")
        W = self.lib.BINARY_FILE_WRITE
        for v in (nx, ny, nz, nvar):
            x = ctypes.c_int(v)
            self._io(W, u, ctypes.byref(x), 1, 4)
        for v in (dt, time):
            x = ctypes.c_double(v)
            self._io(W, u, ctypes.byref(x), 1, 8)
        for n in names:
            b = ctypes.create_string_buffer(n.ljust(8).encode(), 8)
            self._io(W, u, b, 8, 1)
        for v in range(nvar):
            col = np.asfortranarray(data[:, :, :, v])
            self._io(W, u, col.ctypes.data, nx * ny * nz, 8)
        e = ctypes.c_int()
        self.lib.BINARY_FILE_CLOSE(ctypes.byref(u), ctypes.byref(e))

    def read_data(self, path):
        """Header, names and fields in the order data_read reads them: (dims, dt, time, names,
        data (nx, ny, nz, nvar) Fortran order)."""
        u = self._open(path, "r")
        R = self.lib.BINARY_FILE_READ
        dims = np.zeros(4, dtype=np.int32)
        self._io(R, u, dims.ctypes.data, 4, 4)
        dt, time = ctypes.c_double(), ctypes.c_double()
        self._io(R, u, ctypes.byref(dt), 1, 8)
        self._io(R, u, ctypes.byref(time), 1, 8)
        names = []
        for _ in range(int(dims[3])):
            b = ctypes.create_string_buffer(8)
            self._io(R, u, b, 8, 1)
            names.append(b.raw.decode().rstrip(" \x00"))
        nx, ny, nz, nvar = (int(x) for x in dims)
        data = np.zeros((nx, ny, nz, nvar), order="F")
        for v in range(nvar):
            col = np.zeros((nx, ny, nz), order="F")
            self._io(R, u, col.ctypes.data, nx * ny * nz, 8)
            data[:, :, :, v] = col
        e = ctypes.c_int()
        self.lib.BINARY_FILE_CLOSE(ctypes.byref(u), ctypes.byref(e))
        return (nx, ny, nz, nvar), dt.value, time.value, names, data
