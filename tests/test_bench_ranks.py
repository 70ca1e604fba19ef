"""Multi-process logic of bench.py on CPU: two gloo ranks, as torchrun starts them.

Each rank fixes its own replica on its GPU; across ranks there is only the barrier
and the reduction of timing scalars (the slowest rank's time, the sum of units)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    rk = bench.Ranks(backend="gloo")
    rk.barrier()
    # rank r took (r + 1) seconds for 100 * (r + 1) units
    t, n, v = rk.aggregate(float(rank + 1), 100 * (rank + 1))
    q.put((rank, t, n, v, rk.reduce(rank, "MIN")))
    rk.close()


@pytest.mark.timeout(120)
def test_two_ranks_aggregate_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, t, n, v, mn in out:
        assert t == 2.0 and n == 300 and v == 150.0 and mn == 0


def test_single_process_needs_no_process_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    sys.path.insert(0, ROOT)
    import bench

    rk = bench.Ranks()
    assert rk.world == 1 and rk.dist is None
    assert rk.aggregate(2.0, 10) == (2.0, 10, 5.0)
