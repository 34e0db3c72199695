"""The C-ABI library without a GPU: it builds for sm_100a, loads, exports every symbol the
header declares, and refuses to run without a CUDA device (no CPU fallback)."""
import ctypes
import os
import re

import pytest

from tests.conftest import HAS_GPU
from tiger_nga_b200 import build as tbuild
from tiger_nga_b200 import capi

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include")


def declared_functions():
    names = []
    for f in sorted(os.listdir(INCLUDE)):
        if f.endswith(".h"):
            text = open(os.path.join(INCLUDE, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?[\s\*])(tng_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(capi.LIB_PATH):
        tbuild.build(verbose=False)
    return capi.load_library()


def test_header_symbols_exported(lib):
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n


def test_default_cfg_is_reference_defaults(lib):
    cfg = capi.default_cfg()
    assert cfg.rtol == 1e-6 and cfg.atol == 1e-12  # finitechem.f90:266-267
    assert cfg.max_steps == 10000  # finitechem.f90:1025
    assert cfg.precision == capi.TNG_FP64 and cfg.literal_mode == capi.TNG_LIT_REF


def test_bad_arguments_are_errors(lib):
    h = ctypes.c_void_p()
    assert lib.tng_chem_create(b"no-such-mechanism", None, ctypes.byref(h)) == -3
    assert "unknown mechanism" in capi.last_error(lib)
    assert lib.tng_chem_create(None, None, ctypes.byref(h)) == -1


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_no_cpu_fallback_without_device(lib):
    with pytest.raises(capi.ChemError, match="no CUDA device"):
        capi.FiniteChem("grimech30")


def test_new_entry_points_check_arguments_without_a_device(lib):
    """The property, data-file and shim entry points refuse bad arguments on the host, before
    any device work (and without a handle or a GPU)."""
    from tiger_nga_b200.capi import TNG_HOST_PTRS, Extent

    TNG_ERR_ARG = -1  # include/tiger_chem.h

    ext = Extent(imino=1, imaxo=4, jmino=1, jmaxo=1, kmino=1, kmaxo=1, imin=1, imax=4, jmin=1, jmax=1, kmin=1,
                 kmax=1, nscalar=10, isc_sc=1, isc_T=10, isc_H2O=0, isc_CO=0, isc_CO2=0)
    assert lib.tng_chem_density(None, None, None, None, None, ctypes.byref(ext), 1e5, TNG_HOST_PTRS) == TNG_ERR_ARG
    assert lib.tng_chem_transport(None, None, None, None, None, ctypes.byref(ext), None, 0, TNG_HOST_PTRS) == TNG_ERR_ARG
    dims = (ctypes.c_int * 4)()
    assert lib.tng_data_info(b"/nonexistent/tng.bin", dims, None, None, None, 0) == TNG_ERR_ARG
    assert "cannot open" in capi.last_error()
    assert lib.tng_data_read(None, b"/nonexistent/tng.bin", None, 0, None, None, None, 0, 0) == TNG_ERR_ARG  # device, no handle
    # the Fortran-signature shims without a registered handle: no crash, an error message
    lib.tng_set_mechanism_handle(None)
    lib.tng_prodrates_(None, None, None, None, None, None, None)
    assert "no handle registered" in capi.last_error()
    lib.tng_compthermodata_(None, None, None)
    assert "no handle registered" in capi.last_error()
