"""ARTS data files streamed to and from device memory (tng_data_read / tng_data_write with
TNG_DEVICE_PTRS): the same values as the host path, across the 16 MB pinned staging chunks
(a chunk boundary in the middle of a grid line included), and the same file bytes."""
import numpy as np
import pytest

from tiger_nga_b200 import capi

pytestmark = pytest.mark.gpu


def test_device_read_and_write_match_host(tmp_path):
    import torch

    chem = capi.FiniteChem("hydrogen", "fp64")
    dims = (130, 130, 130)
    n = int(np.prod(dims))
    rng = np.random.default_rng(4)
    f = rng.standard_normal((2, n))
    path = str(tmp_path / "big.bin")
    capi.data_write(path, dims, ["T", "RHO"], f, dt=1e-6, time=3.0)
    # whole grid (2.2 M cells per variable: two staging chunks each)
    got = capi.data_read(path, ["RHO", "T"], chem=chem)
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), f[::-1])
    full = f.reshape(2, dims[2], dims[1], dims[0])  # [v][k][j][i]
    # whole lines, chunk boundary inside a line (130 x 128 x 130 = 2,163,200 cells > 2,097,152)
    for start, count in (((0, 1, 0), (130, 128, 130)), ((3, 5, 7), (101, 97, 50)), ((0, 0, 129), (130, 130, 1))):
        got = capi.data_read(path, ["T"], start=start, count=count, chem=chem)
        host = capi.data_read(path, ["T"], start=start, count=count)
        torch.cuda.synchronize()
        (i0, j0, k0), (ci, cj, ck) = start, count
        want = full[0, k0:k0 + ck, j0:j0 + cj, i0:i0 + ci].reshape(-1)
        assert np.array_equal(host[0], want)
        assert np.array_equal(got.cpu().numpy()[0], want)
    # device fields to a file: the same bytes as the host writer
    dev = torch.from_numpy(f).cuda()
    path2 = str(tmp_path / "dev.bin")
    capi.data_write(path2, dims, ["T", "RHO"], dev, dt=1e-6, time=3.0, chem=chem)
    assert open(path2, "rb").read() == open(path, "rb").read()
    chem.close()
