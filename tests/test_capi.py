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
