"""The N>1 path on CPU: bench.py's replica aggregation under gloo with two
ranks.  Each rank advances its own replica of a small case (the oracle stands
in for the device work here), the time is the max over ranks and the job
throughput counts every rank's unknowns."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    import time

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle_api
        from fr_learn_b200 import box2d

        mesh = box2d(4 + rank, 4, -10, 10, -10, 10)  # uneven replicas: times differ
        o = oracle_api.Oracle(oracle_api.params(nDims=2, order=3, riemannType=1, dt=1e-3), mesh)
        o.set_ic(1)
        t0 = time.perf_counter()
        o.update(2)
        ms = (time.perf_counter() - t0) * 1e3 / 2
        dist.barrier()
        mx = bench.max_over_ranks(ms, world)
        q.put((rank, ms, mx, o.nE * o.nS * o.nV))
    finally:
        dist.destroy_process_group()


def test_replica_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    local = [g[1] for g in got]
    reduced = {g[2] for g in got}
    assert len(reduced) == 1 and abs(reduced.pop() - max(local)) < 1e-12


def test_throughput_formula():
    import bench

    assert bench.throughput(4, 1000, 2.0) == pytest.approx(4 * 1000 / 2e-3)
    assert bench.max_over_ranks(3.5, 1) == 3.5
