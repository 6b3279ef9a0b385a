"""The replica plumbing of bench.py on CPU: world size 2 over gloo.

Each rank times a different amount of work; every rank must see the max
over ranks (the bench's timed region), the barrier must release both, and
the reference arm runs on rank 0 only (the other rank does no work).
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as tmp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    D = bench.Dist(world, backend="gloo")
    D.barrier()
    got = D.max(10.0 * (rank + 1))

    class A:
        workload, steps, warmup, pcg_maxiters = "c1", 1, 0, 3000

    ref = bench.run_reference(A(), D) if rank != 0 else "rank0"
    D.barrier()
    D.close()
    out.put((rank, got, ref))


def test_two_ranks_over_gloo():
    world, port = 2, _free_port()
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]  # the max over ranks, on every rank
    assert res[1][2] is None  # the reference arm: rank 1 does no work
