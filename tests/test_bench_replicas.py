"""Replica path of bench.py on CPU: two gloo ranks (world_size 2).

bench.py runs one independent H_eff replica per GPU and reports the whole-job
rate from the slowest rank's device time; this checks the max-over-ranks
reduction, the barrier and the aggregation on the gloo backend, with ranks
that report different times."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = 100.0 + 25.0 * rank  # rank 1 is the slow replica
        m = bench.reduce_max(ms, world)
        q.put((rank, m, bench.replica_rate(world, 10, m)))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, m, rate in res:
        assert m == 125.0
        assert rate == pytest.approx(2 * 10 / 0.125)
