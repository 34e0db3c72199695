"""The multi-GPU plumbing of the benchmark on CPU: two gloo ranks, each owning its own seeded
batch of cells (no data exchange), and the max-over-ranks step time that bench.py reports."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        import bench

        t = bench.max_over_ranks(dist, torch.device("cpu"), 10.0 * (rank + 1))
        wl = dict(bench.WORKLOADS["h2-substep"])
        wl["side"] = 4
        sol, dt = bench.make_state(wl, rank)
        wp = dict(bench.WORKLOADS["gri-transport"])
        wp["side"] = 4
        props, _ = bench.make_state(wp, rank)  # [Y_1..Y_N, T] of this rank's cells
        q.put((rank, t, float(sol.sum()) + float(props[-1].sum()), (sol.shape, props.shape), dt))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_cells_and_report_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, c0, sh0, dt0), (r1, t1, c1, sh1, dt1) = out
    assert t0 == t1 == 20.0            # every rank reports the slowest rank's time
    assert sh0 == sh1 and dt0 == dt1   # same workload shape per rank (weak scaling)
    assert c0 != c1                    # but each rank owns different cells


def _partition_1d(n, nproc, iproc, lo=1):
    """The split of one direction among nproc ranks (iproc 1-based): the first r = n mod nproc
    ranks get q + 1 cells, the rest q (geometry/partition.f90:41-52)."""
    q, r = divmod(n, nproc)
    if iproc <= r:
        return q + 1, lo + (iproc - 1) * (q + 1)
    return q, lo + r * (q + 1) + (iproc - r - 1) * q


def _block_extent(rank, dims, procs, nover, ns, nscalar):
    """This rank's padded block as the host solver's partition_init builds it, as a tng_extent."""
    px, py, pz = procs
    ip, jp, kp = rank % px + 1, (rank // px) % py + 1, rank // (px * py) + 1
    ext = {}
    for (lo_name, hi_name, lo_o, hi_o), n, npr, ipr in zip(
            (("imin", "imax", "imino", "imaxo"), ("jmin", "jmax", "jmino", "jmaxo"), ("kmin", "kmax", "kmino", "kmaxo")),
            dims, procs, (ip, jp, kp)):
        nn, lo = _partition_1d(n, npr, ipr)
        ext[lo_name], ext[hi_name] = lo, lo + nn - 1
        ext[lo_o], ext[hi_o] = lo - nover, lo + nn - 1 + nover
    # species first, then T, then a passive scalar (mixture fraction); H2O at species slot 5
    ext.update(nscalar=nscalar, isc_sc=1, isc_T=ns + 1, isc_H2O=6, isc_CO=0, isc_CO2=0)
    return ext


def _extent_worker(rank, ws, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        from tiger_nga_b200 import capi

        dims, procs, nover, ns = (9, 7, 5), (2, 1, 1), 2, 9
        ext = _block_extent(rank, dims, procs, nover, ns, nscalar=ns + 2)
        plan = capi.extent_plan(ext, ns)
        # the rank's Fortran arrays: SC_(imino:imaxo, jmino:jmaxo, kmino:kmaxo, nscalar), column-major
        shape = tuple(ext[h] - ext[lo] + 1 for lo, h in (("imino", "imaxo"), ("jmino", "jmaxo"), ("kmino", "kmaxo")))
        sc = np.zeros(shape + (ns + 2,), order="F")
        ok_volume = plan["volume"] == sc[..., 0].size
        total = torch.tensor([plan["n_interior"]], dtype=torch.int64)
        dist.all_reduce(total)
        # the host-side checks reject a block whose interior leaves its padded range and a species
        # block that runs past nscalar
        bad = dict(ext, imax=ext["imaxo"] + 1)
        errs = []
        for e in (bad, dict(ext, isc_sc=4)):
            try:
                capi.extent_plan(e, ns)
                errs.append("accepted")
            except capi.ChemError as exc:
                errs.append(str(exc))
        q.put((rank, plan, int(total.item()), ok_volume, errs, (ext["imin"], ext["imax"])))
    finally:
        dist.destroy_process_group()


def test_two_ranks_plan_their_partition_blocks():
    """Each gloo rank builds its own sub-block of a 9x7x5 grid split 2x1x1 with two ghost layers,
    as partition_init does, and drives the substep's host-side extent checks on it (no device):
    the interior cells of the ranks add up to the global grid, each padded volume matches the
    rank's own SC_ array, and inconsistent extents are refused on every rank."""
    pytest.importorskip("numpy")
    from tiger_nga_b200 import capi

    try:
        capi.load_library()
    except capi.ChemError:
        pytest.skip("libtiger_chem.so not built")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_extent_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, plan0, tot0, vol0, errs0, x0), (r1, plan1, tot1, vol1, errs1, x1) = out
    assert tot0 == tot1 == 9 * 7 * 5
    assert plan0["n_interior"] == 5 * 7 * 5 and plan1["n_interior"] == 4 * 7 * 5  # 9 = 5 + 4 along x
    assert x0 == (1, 5) and x1 == (6, 9)
    assert vol0 and vol1
    assert plan0["diag_species"] == plan1["diag_species"] == [5, -1, -1]
    for errs in (errs0, errs1):
        assert "inconsistent extents" in errs[0] and "scalar indices" in errs[1]
