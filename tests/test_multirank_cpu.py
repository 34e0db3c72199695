"""The multi-GPU plumbing of the benchmark on CPU: two gloo ranks, each owning its own seeded
batch of cells (no data exchange), and the max-over-ranks step time that bench.py reports."""
import multiprocessing as mp
import os
import socket

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
