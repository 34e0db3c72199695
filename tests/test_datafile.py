"""ARTS data files (tng_data_info / tng_data_read / tng_data_write, core/data.f90:217-457)
against the reference's own file library (library/fileio_c.c built unchanged into oracle/_ref)
and a golden file it wrote (tests/golden/make_golden_datafile.py). Host paths: no GPU needed."""
import os

import numpy as np
import pytest

from oracle.oracle import REF_FILEIO, RefFileIO
from tiger_nga_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "data_ref_small.bin")


def golden_fields():
    import importlib.util

    spec = importlib.util.spec_from_file_location("mkg", os.path.join(HERE, "golden", "make_golden_datafile.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.fields(), m.NAMES


def test_reads_the_reference_writers_file():
    data, names = golden_fields()
    info = capi.data_info(GOLDEN)
    assert info["dims"] == (5, 4, 3) and info["names"] == names
    assert info["dt"] == 2.5e-6 and info["time"] == 0.125
    got = capi.data_read(GOLDEN, names)
    assert np.array_equal(got, data.reshape(-1, len(names), order="F").T)


@pytest.mark.parametrize("start,count", [((1, 1, 0), (3, 2, 2)), ((0, 0, 1), (5, 4, 2)), ((0, 2, 0), (5, 2, 3)),
                                         ((4, 3, 2), (1, 1, 1))])
def test_sub_blocks_and_variable_order(start, count):
    data, names = golden_fields()
    sel = ["ZMIX", "RHO", "T"]
    got = capi.data_read(GOLDEN, sel, start=start, count=count)
    (i0, j0, k0), (ci, cj, ck) = start, count
    for v, nm in enumerate(sel):
        blk = data[i0:i0 + ci, j0:j0 + cj, k0:k0 + ck, names.index(nm)]
        assert np.array_equal(got[v], blk.reshape(-1, order="F"))


def test_write_then_read_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    dims = (7, 2, 5)
    f = rng.standard_normal((3, int(np.prod(dims))))
    path = str(tmp_path / "d.bin")
    capi.data_write(path, dims, ["U", "V", "SC_01"], f, dt=1e-3, time=2.0)
    info = capi.data_info(path)
    assert info["dims"] == dims and info["names"] == ["U", "V", "SC_01"] and info["time"] == 2.0
    assert np.array_equal(capi.data_read(path, ["U", "V", "SC_01"]), f)
    assert os.path.getsize(path) == 32 + 3 * 8 + 8 * f.size


@pytest.fixture
def short_dir():
    """A directory with a short path: the reference's file library copies names into char[64]."""
    import shutil
    import tempfile

    d = tempfile.mkdtemp(prefix="tng", dir="/tmp")
    yield d
    shutil.rmtree(d, ignore_errors=True)


@pytest.mark.skipif(not os.path.exists(REF_FILEIO), reason="oracle/_ref not built (needs the reference tree)")
def test_reference_reader_reads_our_file_and_writer_matches_bytes(short_dir):
    import pathlib

    tmp_path = pathlib.Path(short_dir)
    data, names = golden_fields()
    ours = str(tmp_path / "ours.bin")
    capi.data_write(ours, data.shape[:3], names, data.reshape(-1, len(names), order="F").T, dt=2.5e-6, time=0.125)
    dims, dt, time, rnames, rdata = RefFileIO().read_data(ours)
    assert dims == (5, 4, 3, 4) and rnames == names and dt == 2.5e-6 and time == 0.125
    assert np.array_equal(rdata, data)
    ref = str(tmp_path / "ref.bin")
    RefFileIO().write_data(ref, data, names, dt=2.5e-6, time=0.125)
    assert open(ours, "rb").read() == open(ref, "rb").read() == open(GOLDEN, "rb").read()


def test_errors(tmp_path):
    with pytest.raises(capi.ChemError):
        capi.data_read(GOLDEN, ["NOPE"])
    with pytest.raises(capi.ChemError):
        capi.data_read(GOLDEN, ["T"], start=(3, 0, 0), count=(3, 1, 1))
    with pytest.raises(capi.ChemError):
        capi.data_write(str(tmp_path / "x.bin"), (2, 2, 2), ["TOO_LONG_NAME"], np.zeros((1, 8)))
    short = tmp_path / "short.bin"
    short.write_bytes(open(GOLDEN, "rb").read()[:100])
    with pytest.raises(capi.ChemError):
        capi.data_info(str(short))
