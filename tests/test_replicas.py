"""The N-GPU replica path: timing reductions over ranks (gloo, 2 processes on CPU).

bench.py --gpus N runs N independent replicas (no halo exchange in the
single-GPU scope); the job time is the maximum over ranks and the throughput
is N times the per-rank units over that time.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from hirep_b200.replicas import max_over_ranks, replica_rate

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = max_over_ranks(1.0 + rank, dist, "cpu")  # rank r took 1 + r ms
        rate = replica_rate(1000.0, t, world)
        out.put((rank, t, rate))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, t, rate in res:
        assert t == pytest.approx(2.0)              # the slowest rank's 2 ms
        assert rate == pytest.approx(2 * 1000 / 2e-3)  # 2 ranks x 1000 units in 2 ms


def test_single_process_needs_no_collective():
    from hirep_b200.replicas import max_over_ranks, replica_rate

    assert max_over_ranks(3.5, None, "cpu") == 3.5
    assert replica_rate(10.0, 2.0, 1) == pytest.approx(5000.0)
