"""Python binding of the C-ABI (``include/tiger_chem.h``) over ctypes.

Mirrors the reference's finite-rate chemistry interface for this path:

* :meth:`FiniteChem.compute_rhs` -- batched ``finitechem_compute_rhs``
  (combustion/finitechem.f90:93-175) with ``PRODRATES`` inside;
* :meth:`FiniteChem.molar_mass`, :attr:`FiniteChem.species`, :attr:`FiniteChem.nspecies`,
  :attr:`FiniteChem.nreactions` -- ``GETMOLARMASS`` / ``GETSPECIESNAMES`` / ``GETNSPECIES`` /
  ``GETNREACTIONS`` (combustion/HYDROGENF.f90:366-450).

The library is the in-tree ``libtiger_chem.so`` built by :mod:`tiger_nga_b200.build`. There is
no CPU fallback: if the library or a CUDA device is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtiger_chem.so")

TNG_FP64, TNG_MIXED = 0, 1
TNG_LIT_REF, TNG_LIT_F64 = 0, 1
TNG_DEVICE_PTRS, TNG_HOST_PTRS = 0, 1


class TngCfg(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("literal_mode", ctypes.c_int), ("device", ctypes.c_int),
                ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("max_steps", ctypes.c_int),
                ("max_newton", ctypes.c_int), ("block_size", ctypes.c_int), ("rate_variant", ctypes.c_int),
                ("solver_warps", ctypes.c_int), ("pass_budget", ctypes.c_int), ("max_passes", ctypes.c_int),
                ("solver_occupancy", ctypes.c_int), ("reserved", ctypes.c_int * 3)]


class SubstepStats(ctypes.Structure):  # noqa: E302
    _fields_ = [("cells", ctypes.c_int64), ("cells_failed", ctypes.c_int64), ("steps", ctypes.c_int64),
                ("newton_iters", ctypes.c_int64), ("jacobians", ctypes.c_int64), ("max_steps_cell", ctypes.c_int),
                ("max_newton_cell", ctypes.c_int), ("passes", ctypes.c_int), ("newton_hist", ctypes.c_int * 16),
                ("ms", ctypes.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "newton_hist"}
        d["newton_hist"] = list(self.newton_hist)
        return d


class SurrogateStats(ctypes.Structure):
    _fields_ = [("cells", ctypes.c_int64), ("accepted", ctypes.c_int64), ("fallback_ood", ctypes.c_int64),
                ("fallback_consistency", ctypes.c_int64), ("fallback_clip", ctypes.c_int64),
                ("judged", ctypes.c_int64), ("judge_max_rel_dT", ctypes.c_double), ("judge_max_dY", ctypes.c_double),
                ("ms_infer", ctypes.c_double), ("ms_post", ctypes.c_double), ("ms_fallback", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("fallback", SubstepStats), ("fallback_ensemble", ctypes.c_int64),
                ("fallback_gate", ctypes.c_int64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "fallback"}
        d["fallback"] = self.fallback.as_dict()
        return d


class SurrogateCfg(ctypes.Structure):
    _fields_ = [("hidden", ctypes.c_int), ("layers", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("ood_margin", ctypes.c_double), ("consist_tol_K", ctypes.c_double), ("clip_tol", ctypes.c_double),
                ("judge_cells", ctypes.c_int), ("post_mode", ctypes.c_int), ("target_mode", ctypes.c_int),
                ("loss_T_weight", ctypes.c_float), ("members", ctypes.c_int), ("ens_tol_K", ctypes.c_float),
                ("ens_tol_Y", ctypes.c_float), ("gate_tol", ctypes.c_float), ("reserved", ctypes.c_int)]


class TuneResult(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("best", ctypes.c_int), ("a", ctypes.c_int * 24), ("b", ctypes.c_int * 24),
                ("ms", ctypes.c_double * 24)]

    def as_list(self):
        return [(self.a[i], self.b[i], self.ms[i]) for i in range(self.n)]


class Extent(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("imino", "imaxo", "jmino", "jmaxo", "kmino", "kmaxo", "imin", "imax",
                                            "jmin", "jmax", "kmin", "kmax", "nscalar", "isc_sc", "isc_T",
                                            "isc_H2O", "isc_CO", "isc_CO2")]


class ChemError(RuntimeError):
    pass


_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load ``libtiger_chem.so`` (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ChemError(f"{p} is missing: build it with `python -m tiger_nga_b200.build` (needs nvcc)")
    lib = ctypes.CDLL(p)
    V, I, D, L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64
    sig = {
        "tng_default_cfg": (None, [ctypes.POINTER(TngCfg)]),
        "tng_last_error": (I, [ctypes.c_char_p, I]),
        "tng_chem_create": (I, [ctypes.c_char_p, ctypes.POINTER(TngCfg), ctypes.POINTER(V)]),
        "tng_chem_destroy": (I, [V]),
        "tng_chem_sizes": (I, [V, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I)]),
        "tng_chem_molar_mass": (I, [V, V]),
        "tng_chem_species_name": (I, [V, I, ctypes.c_char_p, I]),
        "tng_chem_stream": (V, [V]),
        "tng_chem_sync": (I, [V]),
        "tng_prodrates_batch": (I, [V, V, V, L, L, D, I]),
        "tng_prodrates_batch_rates": (I, [V, V, V, V, L, L, D]),
        "tng_bench_fp64_peak": (I, [I, ctypes.POINTER(D)]),
        "tng_substep_batch": (I, [V, V, L, L, V, D, D, I, V, V, V, ctypes.POINTER(SubstepStats)]),
        "tng_solver_rhs_jac": (I, [V, V, L, L, D, V, V]),
        "tng_substep_batch_static": (I, [V, V, L, L, V, D, D, ctypes.POINTER(I)]),
        "tng_surrogate_debug_waits": (I, [V, I, I]),
        "tng_surrogate_refine": (I, [V, V, V, V, L, L, D, I, I, D, D, V, ctypes.POINTER(L)]),
        "tng_surrogate_train_gate": (I, [V, V, V, V, L, L, D, I, I, D, D, V]),
        "tng_surrogate_set_gate_tol": (I, [V, D]),
        "tng_surrogate_gate_info": (I, [V, ctypes.POINTER(I), ctypes.POINTER(D)]),
        "tng_extent_plan": (I, [ctypes.POINTER(Extent), I, ctypes.POINTER(L), ctypes.POINTER(L), ctypes.POINTER(I)]),
        "tng_chem_set_tuning": (I, [V, I, I, I, I]),
        "tng_rates_autotune": (I, [V, V, L, L, D, ctypes.POINTER(TuneResult)]),
        "tng_substep_autotune": (I, [V, V, L, L, V, D, D, L, ctypes.POINTER(TuneResult)]),
        "tng_chem_substep": (I, [V, V, V, V, ctypes.POINTER(Extent), D, D, V, V, I, ctypes.POINTER(SubstepStats)]),
        "tng_chem_density": (I, [V, V, V, V, V, ctypes.POINTER(Extent), D, I]),
        "tng_set_mechanism_handle": (None, [V]),
        "tng_prodrates_": (None, [V, V, V, V, V, ctypes.POINTER(D), ctypes.POINTER(D)]),
        "tng_compthermodata_": (None, [V, V, ctypes.POINTER(D)]),
        "tng_data_info": (I, [ctypes.c_char_p, ctypes.POINTER(I), ctypes.POINTER(D), ctypes.POINTER(D),
                              ctypes.c_char_p, I]),
        "tng_data_read": (I, [V, ctypes.c_char_p, V, I, V, V, V, L, I]),
        "tng_data_write": (I, [V, ctypes.c_char_p, V, V, I, D, D, V, L, I]),
        "tng_chem_transport": (I, [V, V, V, V, V, ctypes.POINTER(Extent), V, I, I]),
        "tng_mlp_create": (I, [V, I, I, I, I, ctypes.c_uint64, ctypes.POINTER(V)]),
        "tng_mlp_destroy": (I, [V]),
        "tng_mlp_param_count": (L, [V]),
        "tng_mlp_get_params": (I, [V, V, I]),
        "tng_mlp_set_params": (I, [V, V]),
        "tng_mlp_forward": (I, [V, V, L, V]),
        "tng_mlp_grad": (I, [V, V, V, V, L, ctypes.POINTER(ctypes.c_float)]),
        "tng_mlp_adam_step": (I, [V, ctypes.c_float]),
        "tng_mlp_set_under_weight": (I, [V, ctypes.c_float]),
        "tng_mlp_train": (I, [V, V, V, V, L, I, I, D, ctypes.c_uint64, V]),
        "tng_surrogate_default_cfg": (None, [ctypes.POINTER(SurrogateCfg)]),
        "tng_surrogate_create": (I, [V, ctypes.POINTER(SurrogateCfg), ctypes.POINTER(V)]),
        "tng_surrogate_destroy": (I, [V]),
        "tng_surrogate_train": (I, [V, V, V, V, L, L, D, I, I, D, V]),
        "tng_surrogate_save": (I, [V, ctypes.c_char_p]),
        "tng_surrogate_load": (I, [V, ctypes.c_char_p]),
        "tng_surrogate_dims": (I, [V, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I),
                                   ctypes.POINTER(L)]),
        "tng_surrogate_params": (I, [V, V, I]),
        "tng_surrogate_features": (I, [V, V, L, L, V, D, V]),
        "tng_surrogate_forward_f32": (I, [V, V, L, V]),
        "tng_surrogate_predict": (I, [V, V, V, L, L, V, D, D, V, L, V, V]),
        "tng_surrogate_infer": (I, [V, V, L, L, V, D, D, V]),
        "tng_substep_surrogate": (I, [V, V, V, L, L, V, D, D, I, ctypes.POINTER(SurrogateStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error(lib=None) -> str:
    lib = lib or load_library()
    buf = ctypes.create_string_buffer(2048)
    lib.tng_last_error(buf, 2048)
    return buf.value.decode()


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise ChemError(f"{what} failed ({rc}): {last_error()}")


def default_cfg() -> TngCfg:
    cfg = TngCfg()
    load_library().tng_default_cfg(ctypes.byref(cfg))
    return cfg


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput of a device (TFLOP/s)."""
    v = ctypes.c_double()
    _check(load_library().tng_bench_fp64_peak(device, ctypes.byref(v)), "tng_bench_fp64_peak")
    return v.value


class FiniteChem:
    """One mechanism on one GPU (a ``tng_chem`` handle and its stream)."""

    def __init__(self, mechanism: str, precision: str = "fp64", literal_mode: str = "ref", device: int = 0,
                 **cfg_fields):
        self.lib = load_library()
        cfg = default_cfg()
        cfg.precision = {"fp64": TNG_FP64, "mixed": TNG_MIXED}[precision]
        cfg.literal_mode = {"ref": TNG_LIT_REF, "f64": TNG_LIT_F64}[literal_mode]
        cfg.device = device
        for k, v in cfg_fields.items():
            setattr(cfg, k, v)
        self.cfg = cfg
        h = ctypes.c_void_p()
        _check(self.lib.tng_chem_create(mechanism.encode(), ctypes.byref(cfg), ctypes.byref(h)), "tng_chem_create")
        self.h = h
        self.mechanism = mechanism
        self.precision = precision
        self.device = device
        ns, nr, nm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.lib.tng_chem_sizes(h, ctypes.byref(ns), ctypes.byref(nr), ctypes.byref(nm)), "tng_chem_sizes")
        self.nspecies, self.nreactions, self.nthirdbody = ns.value, nr.value, nm.value
        self._torch_stream = None
        self._children = weakref.WeakSet()

    def close(self) -> None:
        """Destroy the handle (and first every network/surrogate object created on it)."""
        if getattr(self, "h", None):
            for c in list(getattr(self, "_children", ())):
                c.close()
            self.lib.tng_chem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- mechanism getters -----------------------------------------------------------------
    def molar_mass(self) -> np.ndarray:
        w = np.zeros(self.nspecies)
        _check(self.lib.tng_chem_molar_mass(self.h, w.ctypes.data), "tng_chem_molar_mass")
        return w

    @property
    def species(self) -> list[str]:
        out = []
        buf = ctypes.create_string_buffer(64)
        for k in range(self.nspecies):
            _check(self.lib.tng_chem_species_name(self.h, k, buf, 64), "tng_chem_species_name")
            out.append(buf.value.decode())
        return out

    # ---- streams ---------------------------------------------------------------------------
    def torch_stream(self):
        import torch

        if self._torch_stream is None:
            self._torch_stream = torch.cuda.ExternalStream(self.lib.tng_chem_stream(self.h), device=self.device)
        return self._torch_stream

    def sync(self) -> None:
        _check(self.lib.tng_chem_sync(self.h), "tng_chem_sync")

    # ---- R7: batched right-hand side ------------------------------------------------------
    def compute_rhs(self, sol, p: float, out=None):
        """d(sol)/dt for a species-major batch ``sol`` of shape (N+1, ncells).

        ``sol`` may be a CUDA tensor (device path, asynchronous, ordered with torch's current
        stream) or a NumPy array (host path; copies pipelined through the device).
        """
        nv = self.nspecies + 1
        if isinstance(sol, np.ndarray):
            if sol.dtype != np.float64 or sol.ndim != 2 or sol.shape[0] != nv or not sol.flags.c_contiguous:
                raise ValueError(f"sol must be a C-contiguous float64 array of shape ({nv}, ncells)")
            if out is None:
                out = np.empty_like(sol)
            n = sol.shape[1]
            _check(self.lib.tng_prodrates_batch(self.h, sol.ctypes.data, out.ctypes.data, n, n, float(p),
                                                TNG_HOST_PTRS), "tng_prodrates_batch")
            return out
        import torch

        if not (sol.is_cuda and sol.dtype == torch.float64 and sol.dim() == 2 and sol.shape[0] == nv):
            raise ValueError(f"sol must be a CUDA float64 tensor of shape ({nv}, ncells)")
        if sol.shape[1] > 1 and sol.stride(1) != 1:
            raise ValueError("sol must be species-major with unit stride along cells")
        ld = max(sol.stride(0), sol.shape[1])
        if out is None:
            out = torch.empty_like(sol)
        if sol.shape[1] > 1 and out.stride() != sol.stride():
            raise ValueError("out must have the same strides as sol")
        st = self.torch_stream()
        st.wait_stream(torch.cuda.current_stream(sol.device))
        _check(self.lib.tng_prodrates_batch(self.h, sol.data_ptr(), out.data_ptr(), sol.shape[1], ld, float(p),
                                            TNG_DEVICE_PTRS), "tng_prodrates_batch")
        torch.cuda.current_stream(sol.device).wait_stream(st)
        return out

    def launch_rhs(self, sol_ptr: int, out_ptr: int, ncells: int, ld: int, p: float) -> None:
        """Raw asynchronous launch on the handle's stream (device pointers, no stream joins)."""
        _check(self.lib.tng_prodrates_batch(self.h, sol_ptr, out_ptr, ncells, ld, float(p), TNG_DEVICE_PTRS),
               "tng_prodrates_batch")

    def compute_rhs_rates(self, sol, p: float):
        """compute_rhs plus every slot's rate W_r (device tensors; reference literal kinds only)."""
        import torch

        nv = self.nspecies + 1
        n = sol.shape[1]
        if sol.stride(1) != 1 or sol.shape[0] != nv:
            raise ValueError("sol must be species-major (N+1, ncells)")
        out = torch.empty_like(sol)
        rates = torch.empty((self.nreactions, n), dtype=torch.float64, device=sol.device)
        if sol.stride(0) != n:
            raise ValueError("compute_rhs_rates needs a dense batch (ld == ncells)")
        st = self.torch_stream()
        st.wait_stream(torch.cuda.current_stream(sol.device))
        _check(self.lib.tng_prodrates_batch_rates(self.h, sol.data_ptr(), out.data_ptr(), rates.data_ptr(), n, n,
                                                  float(p)), "tng_prodrates_batch_rates")
        torch.cuda.current_stream(sol.device).wait_stream(st)
        return out, rates


def _substep(self, state, dt, p: float, cell_counts: bool = False, stats: bool = True):
    """The implicit chemistry substep (finitechem_source_chemistry's per-cell integration).

    ``state`` is a species-major (N+1, ncells) batch of (rho*Y_k, rho*T), advanced in place over
    ``dt`` (a scalar or a per-cell array/tensor). CUDA tensors stay on the device; NumPy arrays
    go through the host-pointer path. Returns the statistics dict (and per-cell counters when
    ``cell_counts``).
    """
    nv = self.nspecies + 1
    st = SubstepStats()
    stp = ctypes.byref(st) if stats else None
    if isinstance(state, np.ndarray):
        if state.dtype != np.float64 or state.ndim != 2 or state.shape[0] != nv or not state.flags.c_contiguous:
            raise ValueError(f"state must be a C-contiguous float64 array of shape ({nv}, ncells)")
        n = state.shape[1]
        dts = None
        if np.ndim(dt):
            dts = np.ascontiguousarray(dt, dtype=np.float64)
            if dts.shape != (n,):
                raise ValueError("per-cell dt must have shape (ncells,)")
        _check(self.lib.tng_substep_batch(self.h, state.ctypes.data, n, n, dts.ctypes.data if dts is not None else None,
                                          0.0 if dts is not None else float(dt), float(p), TNG_HOST_PTRS, None, None,
                                          None, stp), "tng_substep_batch")
        return st.as_dict() if stats else None
    import torch

    if not (state.is_cuda and state.dtype == torch.float64 and state.dim() == 2 and state.shape[0] == nv):
        raise ValueError(f"state must be a CUDA float64 tensor of shape ({nv}, ncells)")
    n = state.shape[1]
    if n > 1 and state.stride(1) != 1:
        raise ValueError("state must be species-major with unit stride along cells")
    ld = max(state.stride(0), n)
    dts = None
    if not isinstance(dt, (float, int)):
        dts = torch.as_tensor(dt, dtype=torch.float64, device=state.device).contiguous()
        if dts.shape != (n,):
            raise ValueError("per-cell dt must have shape (ncells,)")
    cnt = None
    if cell_counts:
        cnt = torch.zeros((3, n), dtype=torch.int32, device=state.device)
    sst = self.torch_stream()
    sst.wait_stream(torch.cuda.current_stream(state.device))
    _check(self.lib.tng_substep_batch(self.h, state.data_ptr(), n, ld, dts.data_ptr() if dts is not None else None,
                                      0.0 if dts is not None else float(dt), float(p), TNG_DEVICE_PTRS,
                                      cnt[0].data_ptr() if cnt is not None else None,
                                      cnt[1].data_ptr() if cnt is not None else None,
                                      cnt[2].data_ptr() if cnt is not None else None, stp), "tng_substep_batch")
    torch.cuda.current_stream(state.device).wait_stream(sst)
    out = st.as_dict() if stats else None
    if cell_counts:
        return out, {"nst": cnt[0], "nni": cnt[1], "status": cnt[2]}
    return out


def _solver_rhs_jac(self, state, p: float, jacobian: bool = True):
    """The solver's own right-hand side and Jacobian (parity helper), CUDA tensors."""
    import torch

    nv = self.nspecies + 1
    n = state.shape[1]
    if state.stride(1) != 1 and n > 1:
        raise ValueError("state must be species-major")
    rhs = torch.empty((nv, n), dtype=torch.float64, device=state.device)
    jac = torch.empty((n, nv, nv), dtype=torch.float64, device=state.device) if jacobian else None
    if state.stride(0) != n:
        state = state.contiguous()
    sst = self.torch_stream()
    sst.wait_stream(torch.cuda.current_stream(state.device))
    _check(self.lib.tng_solver_rhs_jac(self.h, state.data_ptr(), n, n, float(p), rhs.data_ptr(),
                                       jac.data_ptr() if jac is not None else None), "tng_solver_rhs_jac")
    torch.cuda.current_stream(state.device).wait_stream(sst)
    return rhs, jac


def _source_chemistry(self, RHO, SC, ext: dict, dt: float, p_mid: float, mask=None, HR=None, chemsrc=None):
    """finitechem_source_chemistry(RHO_, SC_) on the solver's own arrays (NumPy, Fortran order)."""
    for a in (RHO, SC):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.f_contiguous):
            raise ValueError("RHO and SC must be Fortran-ordered float64 arrays")
    e = Extent(**ext)
    st = SubstepStats()
    mk = None
    if mask is not None:
        mk = np.asfortranarray(mask, dtype=np.int32)
    _check(self.lib.tng_chem_substep(self.h, RHO.ctypes.data, SC.ctypes.data, mk.ctypes.data if mk is not None else None,
                                     ctypes.byref(e), float(dt), float(p_mid), HR.ctypes.data if HR is not None else None,
                                     chemsrc.ctypes.data if chemsrc is not None else None, TNG_HOST_PTRS,
                                     ctypes.byref(st)), "tng_chem_substep")
    return st.as_dict()


def _fortran_f64(*arrays):
    for a in arrays:
        if a is not None and not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.f_contiguous):
            raise ValueError("arrays must be Fortran-ordered float64 NumPy arrays")


def _density(self, RHO, SC, ext: dict, p_thermo: float, mask=None, W=None):
    """finitechem_density (finitechem.f90:324-345) on the solver's own arrays (NumPy, Fortran
    order): RHO (and W_mix into W when given) for every unmasked cell of the padded block."""
    _fortran_f64(RHO, SC, W)
    e = Extent(**ext)
    mk = None if mask is None else np.asfortranarray(mask, dtype=np.int32)
    _check(self.lib.tng_chem_density(self.h, RHO.ctypes.data if RHO is not None else None,
                                     W.ctypes.data if W is not None else None, SC.ctypes.data,
                                     mk.ctypes.data if mk is not None else None, ctypes.byref(e), float(p_thermo),
                                     TNG_HOST_PTRS), "tng_chem_density")


def _transport(self, SC, ext: dict, VISC=None, DIFF=None, mask=None, lewis=None, isc_zmix: int = 0):
    """finitechem_viscosity + finitechem_diffusivity (finitechem.f90:351-461) on the solver's own
    arrays: VISC shaped like RHO, DIFF shaped like SC (species, T and ZMIX columns written)."""
    _fortran_f64(SC, VISC, DIFF)
    e = Extent(**ext)
    mk = None if mask is None else np.asfortranarray(mask, dtype=np.int32)
    lw = None if lewis is None else np.ascontiguousarray(lewis, dtype=np.float64)
    _check(self.lib.tng_chem_transport(self.h, VISC.ctypes.data if VISC is not None else None,
                                       DIFF.ctypes.data if DIFF is not None else None, SC.ctypes.data,
                                       mk.ctypes.data if mk is not None else None, ctypes.byref(e),
                                       lw.ctypes.data if lw is not None else None, int(isc_zmix), TNG_HOST_PTRS),
           "tng_chem_transport")


def batch_extent(ncells: int, nspecies: int) -> Extent:
    """The extent that presents a species-major device batch [Y_1..Y_N, T] (shape (N+1, ncells))
    as a one-row Fortran block: nscalar N+1, species at 1..N, T at N+1."""
    return Extent(imino=1, imaxo=ncells, jmino=1, jmaxo=1, kmino=1, kmaxo=1, imin=1, imax=ncells, jmin=1, jmax=1,
                  kmin=1, kmax=1, nscalar=nspecies + 1, isc_sc=1, isc_T=nspecies + 1, isc_H2O=0, isc_CO=0, isc_CO2=0)


def _mixture_props(self, sc, p_thermo: float | None = None, visc: bool = False, diff: bool = False, lewis=None,
                   out=None):
    """Mixture properties of a species-major CUDA batch ``sc`` = [Y_1..Y_N, T] (float64, shape
    (N+1, ncells), unit stride along cells): with p_thermo, 'rho' and 'wmix' (tng_chem_density);
    with visc / diff, 'visc' (ncells) and 'diff' ((N+1, ncells): lambda/Cp_mix/Lewis_k, then
    lambda/Cp_mix) from tng_chem_transport. ``out`` may supply the output tensors."""
    import torch

    ns = self.nspecies
    if not (sc.is_cuda and sc.dtype == torch.float64 and sc.dim() == 2 and sc.shape[0] == ns + 1 and sc.is_contiguous()):
        raise ValueError(f"sc must be a contiguous CUDA float64 tensor of shape ({ns + 1}, ncells)")
    n = sc.shape[1]
    e = batch_extent(n, ns)
    out = dict(out or {})
    sst = self.torch_stream()
    sst.wait_stream(torch.cuda.current_stream(sc.device))
    if p_thermo is not None:
        for k in ("rho", "wmix"):
            out.setdefault(k, torch.empty(n, dtype=torch.float64, device=sc.device))
        _check(self.lib.tng_chem_density(self.h, out["rho"].data_ptr(), out["wmix"].data_ptr(), sc.data_ptr(), None,
                                         ctypes.byref(e), float(p_thermo), TNG_DEVICE_PTRS), "tng_chem_density")
    if visc or diff:
        if visc:
            out.setdefault("visc", torch.empty(n, dtype=torch.float64, device=sc.device))
        if diff:
            out.setdefault("diff", torch.empty((ns + 1, n), dtype=torch.float64, device=sc.device))
        lw = None if lewis is None else np.ascontiguousarray(lewis, dtype=np.float64)
        _check(self.lib.tng_chem_transport(self.h, out["visc"].data_ptr() if visc else None,
                                           out["diff"].data_ptr() if diff else None, sc.data_ptr(), None,
                                           ctypes.byref(e), lw.ctypes.data if lw is not None else None, 0,
                                           TNG_DEVICE_PTRS), "tng_chem_transport")
    torch.cuda.current_stream(sc.device).wait_stream(sst)
    return out


def extent_plan(ext: dict, nspecies: int) -> dict:
    """tng_extent_plan: host-side checks of a rank's padded block (no device needed). Returns
    the interior cell count, the padded volume and the H2O / CO / CO2 species positions."""
    lib = load_library()
    e = Extent(**ext)
    n, vol = ctypes.c_int64(), ctypes.c_int64()
    sp = (ctypes.c_int * 3)()
    _check(lib.tng_extent_plan(ctypes.byref(e), int(nspecies), ctypes.byref(n), ctypes.byref(vol), sp),
           "tng_extent_plan")
    return {"n_interior": n.value, "volume": vol.value, "diag_species": list(sp)}


def _names(vars_):
    arr = (ctypes.c_char_p * len(vars_))(*[v.encode() for v in vars_])
    return arr


def data_info(path: str) -> dict:
    """Header of an ARTS data file (tng_data_info): dims, dt, time, variable names."""
    lib = load_library()
    dims = (ctypes.c_int * 4)()
    dt, time = ctypes.c_double(), ctypes.c_double()
    _check(lib.tng_data_info(path.encode(), dims, ctypes.byref(dt), ctypes.byref(time), None, 0), "tng_data_info")
    buf = ctypes.create_string_buffer(8 * dims[3] + 1)
    _check(lib.tng_data_info(path.encode(), dims, None, None, buf, 8 * dims[3] + 1), "tng_data_info")
    raw = buf.raw[:8 * dims[3]].decode()
    return {"dims": tuple(dims[:3]), "nvars": dims[3], "dt": dt.value, "time": time.value,
            "names": [raw[8 * v:8 * v + 8].rstrip() for v in range(dims[3])]}


def data_read(path: str, vars_, start=None, count=None, chem: "FiniteChem | None" = None, out=None):
    """The named variables of a sub-block (0-based start / count along i, j, k; default the whole
    grid) of an ARTS data file (tng_data_read), species-major (nvar, ncells of the block, i
    fastest). With ``chem`` the result is a CUDA tensor on its device, else a NumPy array."""
    lib = load_library()
    info = data_info(path)
    s = list(start) if start is not None else [0, 0, 0]
    c = list(count) if count is not None else [d - o for d, o in zip(info["dims"], s)]
    n = int(np.prod(c))
    si, ci = (ctypes.c_int * 3)(*s), (ctypes.c_int * 3)(*c)
    if chem is None:
        out = np.empty((len(vars_), n)) if out is None else out
        _check(lib.tng_data_read(None, path.encode(), _names(vars_), len(vars_), si, ci, out.ctypes.data, n,
                                 TNG_HOST_PTRS), "tng_data_read")
        return out
    import torch

    out = torch.empty((len(vars_), n), dtype=torch.float64, device=f"cuda:{chem.device}") if out is None else out
    chem.torch_stream().wait_stream(torch.cuda.current_stream(out.device))
    _check(lib.tng_data_read(chem.h, path.encode(), _names(vars_), len(vars_), si, ci, out.data_ptr(), n,
                             TNG_DEVICE_PTRS), "tng_data_read")
    return out


def data_write(path: str, dims, vars_, fields, dt: float = 0.0, time: float = 0.0, chem: "FiniteChem | None" = None):
    """Write an ARTS data file of the whole grid dims = (nx, ny, nz) (tng_data_write); fields is
    (nvar, nx*ny*nz), i fastest: a NumPy array, or a CUDA tensor with ``chem``."""
    lib = load_library()
    d = (ctypes.c_int * 3)(*dims)
    n = int(np.prod(dims))
    if chem is None:
        f = np.ascontiguousarray(fields, dtype=np.float64)
        _check(lib.tng_data_write(None, path.encode(), d, _names(vars_), len(vars_), float(dt), float(time),
                                  f.ctypes.data, n, TNG_HOST_PTRS), "tng_data_write")
        return
    import torch

    chem.torch_stream().wait_stream(torch.cuda.current_stream(fields.device))
    _check(lib.tng_data_write(chem.h, path.encode(), d, _names(vars_), len(vars_), float(dt), float(time),
                              fields.contiguous().data_ptr(), n, TNG_DEVICE_PTRS), "tng_data_write")


def _prodrates_cell(self, C, T: float, P: float):
    """One cell through the Fortran-signature shim tng_prodrates_ (PRODRATES(CDOT, W, K, C, M, T, P)):
    returns (CDOT [kmol/m^3/s], W slot rates)."""
    c = np.ascontiguousarray(C, dtype=np.float64)
    cdot, w = np.zeros(self.nspecies), np.zeros(self.nreactions)
    k, m = np.zeros(self.nreactions), np.zeros(max(self.nthirdbody, 1))
    self.lib.tng_set_mechanism_handle(self.h)
    self.lib.tng_prodrates_(cdot.ctypes.data, w.ctypes.data, k.ctypes.data, c.ctypes.data, m.ctypes.data,
                            ctypes.byref(ctypes.c_double(T)), ctypes.byref(ctypes.c_double(P)))
    if np.isnan(cdot).any():
        raise ChemError(f"tng_prodrates_ failed: {last_error()}")
    return cdot, w


def _thermo_cell(self, T: float):
    """COMPTHERMODATA(H, CP, T) through the shim tng_compthermodata_: (h [J/kg], cp [J/(kg K)])."""
    hk, cp = np.zeros(self.nspecies), np.zeros(self.nspecies)
    self.lib.tng_set_mechanism_handle(self.h)
    self.lib.tng_compthermodata_(hk.ctypes.data, cp.ctypes.data, ctypes.byref(ctypes.c_double(T)))
    if np.isnan(hk).any():
        raise ChemError(f"tng_compthermodata_ failed: {last_error()}")
    return hk, cp


def _substep_static(self, state, dt, p: float) -> int:
    """tng_substep_batch_static on a CUDA tensor (allocates nothing on the device during the
    call; at most 262144 cells; calls must not overlap). Returns the number of failed cells."""
    import torch

    nv = self.nspecies + 1
    if not (state.is_cuda and state.dtype == torch.float64 and state.dim() == 2 and state.shape[0] == nv):
        raise ValueError(f"state must be a CUDA float64 tensor of shape ({nv}, ncells)")
    n = state.shape[1]
    if n > 1 and state.stride(1) != 1:
        raise ValueError("state must be species-major with unit stride along cells")
    dts = None
    if not isinstance(dt, (float, int)):
        dts = torch.as_tensor(dt, dtype=torch.float64, device=state.device).contiguous()
        if dts.shape != (n,):
            raise ValueError("per-cell dt must have shape (ncells,)")
    failed = ctypes.c_int(0)
    sst = self.torch_stream()
    sst.wait_stream(torch.cuda.current_stream(state.device))
    _check(self.lib.tng_substep_batch_static(self.h, state.data_ptr(), n, max(state.stride(0), n),
                                             dts.data_ptr() if dts is not None else None,
                                             0.0 if dts is not None else float(dt), float(p), ctypes.byref(failed)),
           "tng_substep_batch_static")
    torch.cuda.current_stream(state.device).wait_stream(sst)
    return failed.value


def _tuning_key(self, kind: str) -> str:
    import torch

    return f"{kind}/{self.mechanism}/{self.precision}/{torch.cuda.get_device_name()}"


def _autotune(self, state, dt=None, p: float = 101325.0, kind: str = "substep", sample: int = 65536,
              cache: str | None = None):
    """Run the project's autotuner on ``state`` (a CUDA tensor of the caller's cells) and keep the
    fastest launch configuration in the handle. kind 'rates' times the rate kernel's variants x
    block sizes; 'substep' times the implicit solver's cells-per-block x pass budget on a sample.
    With ``cache`` (a JSON file) a stored choice for this mechanism, precision and GPU is applied
    without timing, and a new one is stored. Returns {"best": (a, b), "candidates": [(a, b, ms)]}."""
    import json
    import os

    import torch

    key = self._tuning_key(kind)
    store = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            store = json.load(f)
        if key in store:
            a, b = store[key]["best"]
            if kind == "rates":
                _check(self.lib.tng_chem_set_tuning(self.h, a, b, self.cfg.solver_warps, self.cfg.pass_budget),
                       "tng_chem_set_tuning")
                self.cfg.rate_variant, self.cfg.block_size = a, b
            else:
                _check(self.lib.tng_chem_set_tuning(self.h, self.cfg.rate_variant, self.cfg.block_size, a, b),
                       "tng_chem_set_tuning")
                self.cfg.solver_warps, self.cfg.solver_occupancy = (8, 2) if a == 16 else (a, 1)
                self.cfg.pass_budget = b
            return store[key]
    n = state.shape[1]
    ld = max(state.stride(0), n)
    res = TuneResult()
    sst = self.torch_stream()
    sst.wait_stream(torch.cuda.current_stream(state.device))
    if kind == "rates":
        _check(self.lib.tng_rates_autotune(self.h, state.data_ptr(), n, ld, float(p), ctypes.byref(res)),
               "tng_rates_autotune")
    else:
        dts = None
        if dt is not None and not isinstance(dt, (float, int)):
            dts = torch.as_tensor(dt, dtype=torch.float64, device=state.device).contiguous()
        _check(self.lib.tng_substep_autotune(self.h, state.data_ptr(), n, ld, dts.data_ptr() if dts is not None else None,
                                             0.0 if dts is not None else float(dt), float(p), int(sample),
                                             ctypes.byref(res)), "tng_substep_autotune")
    a, b = res.a[res.best], res.b[res.best]
    if kind == "rates":
        self.cfg.rate_variant, self.cfg.block_size = a, b
    else:
        self.cfg.solver_warps, self.cfg.solver_occupancy = (8, 2) if a == 16 else (a, 1)
        self.cfg.pass_budget = b
    out = {"best": (a, b), "candidates": res.as_list()}
    if cache:
        store[key] = out
        with open(cache, "w") as f:
            json.dump(store, f, indent=1)
    return out


FiniteChem._tuning_key = _tuning_key
FiniteChem.autotune = _autotune
FiniteChem.source_chemistry = _source_chemistry
FiniteChem.prodrates_cell = _prodrates_cell
FiniteChem.thermo_cell = _thermo_cell
FiniteChem.density = _density
FiniteChem.transport = _transport
FiniteChem.mixture_props = _mixture_props
FiniteChem.substep_static = _substep_static
FiniteChem.substep = _substep
FiniteChem.solver_rhs_jac = _solver_rhs_jac


class Mlp:
    """The surrogate network on the device of a FiniteChem handle (tng_mlp_*)."""

    def __init__(self, chem: "FiniteChem", n_in: int, n_out: int, hidden: int = 256, layers: int = 4, seed: int = 0):
        self.lib = chem.lib
        self.chem = chem
        h = ctypes.c_void_p()
        _check(self.lib.tng_mlp_create(chem.h, n_in, n_out, hidden, layers, seed, ctypes.byref(h)), "tng_mlp_create")
        self.h = h
        self.n_in, self.n_out, self.hidden, self.layers = n_in, n_out, hidden, layers
        self.in_pad, self.out_pad = -(-n_in // 16) * 16, -(-n_out // 16) * 16
        self.nparam = self.lib.tng_mlp_param_count(h)
        chem._children.add(self)

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.chem, "h", None):
                self.lib.tng_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shapes(self):
        out, fi = [], self.in_pad
        for l in range(self.layers + 1):
            fo = self.out_pad if l == self.layers else self.hidden
            out.append(((fo, fi), (fo,)))
            fi = fo
        return out

    def get(self, which: int = 0):
        buf = np.zeros(self.nparam, dtype=np.float32)
        _check(self.lib.tng_mlp_get_params(self.h, buf.ctypes.data, which), "tng_mlp_get_params")
        return self.unflatten(buf)

    def unflatten(self, buf):
        out, off = [], 0
        for (ws, bs) in self.shapes():
            nw = ws[0] * ws[1]
            W = buf[off:off + nw].reshape(ws)
            off += nw
            b = buf[off:off + bs[0]]
            off += bs[0]
            out.append((W, b))
        return out

    def set(self, params):
        flat = np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in params]).astype(np.float32)
        _check(self.lib.tng_mlp_set_params(self.h, flat.ctypes.data), "tng_mlp_set_params")

    def _dev(self, a, width):
        import torch

        t = torch.as_tensor(a, dtype=torch.float32, device=f"cuda:{self.chem.device}").contiguous()
        if t.dim() != 2 or t.shape[1] != width:
            raise ValueError(f"expected (rows, {width})")
        return t

    def forward(self, X):
        import torch

        Xd = self._dev(X, self.in_pad)
        Y = torch.empty((Xd.shape[0], self.out_pad), dtype=torch.float32, device=Xd.device)
        self._sync_in()
        _check(self.lib.tng_mlp_forward(self.h, Xd.data_ptr(), Xd.shape[0], Y.data_ptr()), "tng_mlp_forward")
        self._sync_out()
        return Y

    def grad(self, X, T, w_out):
        Xd, Td = self._dev(X, self.in_pad), self._dev(T, self.out_pad)
        wd = self._dev(np.asarray(w_out, dtype=np.float32)[None, :], self.out_pad)
        loss = ctypes.c_float()
        self._sync_in()
        _check(self.lib.tng_mlp_grad(self.h, Xd.data_ptr(), Td.data_ptr(), wd.data_ptr(), Xd.shape[0],
                                     ctypes.byref(loss)), "tng_mlp_grad")
        return loss.value, self.get(1)

    def adam_step(self, lr):
        _check(self.lib.tng_mlp_adam_step(self.h, float(lr)), "tng_mlp_adam_step")

    def set_under_weight(self, under: float):
        """Weight of squared errors of outputs below their target (1: plain weighted MSE)."""
        _check(self.lib.tng_mlp_set_under_weight(self.h, float(under)), "tng_mlp_set_under_weight")

    def train(self, X, T, w_out, epochs, batch, lr, seed=0):
        Xd, Td = self._dev(X, self.in_pad), self._dev(T, self.out_pad)
        wd = self._dev(np.asarray(w_out, dtype=np.float32)[None, :], self.out_pad)
        losses = np.zeros(epochs, dtype=np.float32)
        self._sync_in()
        _check(self.lib.tng_mlp_train(self.h, Xd.data_ptr(), Td.data_ptr(), wd.data_ptr(), Xd.shape[0], epochs, batch,
                                      float(lr), seed, losses.ctypes.data), "tng_mlp_train")
        return losses

    def _sync_in(self):
        import torch

        self.chem.torch_stream().wait_stream(torch.cuda.current_stream(self.chem.device))

    def _sync_out(self):
        import torch

        torch.cuda.current_stream(self.chem.device).wait_stream(self.chem.torch_stream())


class Surrogate:
    """The learned substep with fallback (tng_surrogate_*), bound to a FiniteChem handle."""

    def __init__(self, chem: "FiniteChem", **cfg_fields):
        self.lib = chem.lib
        self.chem = chem
        cfg = SurrogateCfg()
        self.lib.tng_surrogate_default_cfg(ctypes.byref(cfg))
        for k, v in cfg_fields.items():
            setattr(cfg, k, v)
        self.cfg = cfg
        h = ctypes.c_void_p()
        _check(self.lib.tng_surrogate_create(chem.h, ctypes.byref(cfg), ctypes.byref(h)), "tng_surrogate_create")
        self.h = h
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        n = ctypes.c_int64()
        _check(self.lib.tng_surrogate_dims(h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d),
                                           ctypes.byref(n)), "tng_surrogate_dims")
        self.n_in, self.n_out, self.in_pad, self.out_pad, self.nparam = a.value, b.value, c.value, d.value, n.value
        self.members = cfg.members
        H, nh = cfg.hidden, cfg.layers
        # weights (no biases) of the linear layers n_in -> H -> ... -> H -> n_out, and as executed
        # with the inputs and outputs padded to the tensor-core tile
        self.weights_unpadded = self.n_in * H + (nh - 1) * H * H + H * self.n_out
        self.weights_padded = self.in_pad * H + (nh - 1) * H * H + H * self.out_pad
        chem._children.add(self)

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.chem, "h", None):
                self.lib.tng_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _pre(self):
        import torch

        self.chem.torch_stream().wait_stream(torch.cuda.current_stream(self.chem.device))

    def _post(self):
        import torch

        torch.cuda.current_stream(self.chem.device).wait_stream(self.chem.torch_stream())

    def train(self, state0, state1, dts, p: float, epochs: int = 10, batch: int = 4096, lr: float = 1e-3):
        """Fit on implicit-solver pairs (CUDA float64 tensors, species-major)."""
        n = state0.shape[1]
        losses = np.zeros(epochs, dtype=np.float32)
        self._pre()
        _check(self.lib.tng_surrogate_train(self.h, state0.data_ptr(), state1.data_ptr(), dts.data_ptr(), n,
                                            state0.stride(0), float(p), epochs, batch, float(lr), losses.ctypes.data),
               "tng_surrogate_train")
        self._post()
        return losses

    def refine(self, state0, state1, dts, p: float, epochs: int = 10, batch: int = 4096, lr: float = 3e-4,
               boost: float = 4.0):
        """Hard-example refinement: more epochs on a population where each pair repeats by its error."""
        losses = np.zeros(epochs, dtype=np.float32)
        pop = ctypes.c_int64()
        self._pre()
        _check(self.lib.tng_surrogate_refine(self.h, state0.data_ptr(), state1.data_ptr(), dts.data_ptr(),
                                             state0.shape[1], state0.stride(0), float(p), epochs, batch, float(lr),
                                             float(boost), losses.ctypes.data, ctypes.byref(pop)),
               "tng_surrogate_refine")
        self._post()
        return losses, pop.value

    def train_gate(self, state0, state1, dts, p: float, epochs: int = 10, batch: int = 4096, lr: float = 2e-3,
                   under: float = 4.0):
        """Train the error gate on implicit-solver pairs (the ensemble's own errors as targets)."""
        losses = np.zeros(epochs, dtype=np.float32)
        self._pre()
        _check(self.lib.tng_surrogate_train_gate(self.h, state0.data_ptr(), state1.data_ptr(), dts.data_ptr(),
                                                 state0.shape[1], state0.stride(0), float(p), epochs, batch,
                                                 float(lr), float(under), losses.ctypes.data),
               "tng_surrogate_train_gate")
        self._post()
        return losses

    def set_gate_tol(self, tol: float):
        _check(self.lib.tng_surrogate_set_gate_tol(self.h, float(tol)), "tng_surrogate_set_gate_tol")

    def gate_info(self):
        g, t = ctypes.c_int(), ctypes.c_double()
        _check(self.lib.tng_surrogate_gate_info(self.h, ctypes.byref(g), ctypes.byref(t)), "tng_surrogate_gate_info")
        return bool(g.value), t.value

    def save(self, path: str):
        _check(self.lib.tng_surrogate_save(self.h, path.encode()), "tng_surrogate_save")

    def load(self, path: str):
        _check(self.lib.tng_surrogate_load(self.h, path.encode()), "tng_surrogate_load")

    def params(self):
        buf = np.zeros(self.nparam, dtype=np.float32)
        _check(self.lib.tng_surrogate_params(self.h, buf.ctypes.data, 0), "tng_surrogate_params")
        return buf

    def features(self, state, dts, p: float):
        import torch

        n = state.shape[1]
        X = torch.empty((n, self.in_pad), dtype=torch.float32, device=state.device)
        self._pre()
        _check(self.lib.tng_surrogate_features(self.h, state.data_ptr(), n, state.stride(0), dts.data_ptr(), float(p),
                                               X.data_ptr()), "tng_surrogate_features")
        return X

    def predict(self, state, dt, p: float):
        """Post-processed prediction of every cell (no fallback): (out state, reason, indicator K)."""
        import torch

        n = state.shape[1]
        dts = None if isinstance(dt, (float, int)) else torch.as_tensor(dt, dtype=torch.float64,
                                                                        device=state.device).contiguous()
        out = torch.empty((state.shape[0], n), dtype=torch.float64, device=state.device)
        reason = torch.empty(n, dtype=torch.int32, device=state.device)
        ind = torch.empty((n, 5), dtype=torch.float64, device=state.device)
        self._pre()
        _check(self.lib.tng_surrogate_predict(self.chem.h, self.h, state.data_ptr(), n, max(state.stride(0), n),
                                              dts.data_ptr() if dts is not None else None,
                                              0.0 if dts is not None else float(dt), float(p), out.data_ptr(), n,
                                              reason.data_ptr(), ind.data_ptr()), "tng_surrogate_predict")
        self._post()
        return out, reason, ind

    def debug_waits(self, wait_limit: int = 0, fault: int = 0):
        """Test hook: later inferences give up a wait after ``wait_limit`` polls; ``fault=1``
        withholds one completion signal so the wait runs out (TNG_ERR_CUDA). (0, 0) resets."""
        _check(self.lib.tng_surrogate_debug_waits(self.h, int(wait_limit), int(fault)), "tng_surrogate_debug_waits")

    def forward_f32(self, X):
        import torch

        Y = torch.empty((X.shape[0], self.out_pad), dtype=torch.float32, device=X.device)
        self._pre()
        _check(self.lib.tng_surrogate_forward_f32(self.h, X.data_ptr(), X.shape[0], Y.data_ptr()),
               "tng_surrogate_forward_f32")
        return Y

    def infer(self, state, dts, p: float):
        import torch

        n = state.shape[1]
        Y = torch.empty((n, self.out_pad), dtype=torch.float32, device=state.device)
        self._pre()
        _check(self.lib.tng_surrogate_infer(self.h, state.data_ptr(), n, state.stride(0), dts.data_ptr(), 0.0,
                                            float(p), Y.data_ptr()), "tng_surrogate_infer")
        self._post()
        return Y

    def substep(self, state, dt, p: float):
        """The substep through the surrogate with fallback; state advanced in place. Returns stats."""
        st = SurrogateStats()
        nv = self.chem.nspecies + 1
        if isinstance(state, np.ndarray):
            n = state.shape[1]
            if state.shape[0] != nv or not state.flags.c_contiguous or state.dtype != np.float64:
                raise ValueError("state must be C-contiguous float64 (N+1, ncells)")
            dts = np.ascontiguousarray(dt, dtype=np.float64) if np.ndim(dt) else None
            _check(self.lib.tng_substep_surrogate(self.chem.h, self.h, state.ctypes.data, n, n,
                                                  dts.ctypes.data if dts is not None else None,
                                                  0.0 if dts is not None else float(dt), float(p), TNG_HOST_PTRS,
                                                  ctypes.byref(st)), "tng_substep_surrogate")
            return st.as_dict()
        import torch

        n = state.shape[1]
        dts = None
        if not isinstance(dt, (float, int)):
            dts = torch.as_tensor(dt, dtype=torch.float64, device=state.device).contiguous()
        self._pre()
        _check(self.lib.tng_substep_surrogate(self.chem.h, self.h, state.data_ptr(), n, max(state.stride(0), n),
                                              dts.data_ptr() if dts is not None else None,
                                              0.0 if dts is not None else float(dt), float(p), TNG_DEVICE_PTRS,
                                              ctypes.byref(st)), "tng_substep_surrogate")
        self._post()
        return st.as_dict()
