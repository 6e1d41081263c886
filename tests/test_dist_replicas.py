"""Multi-GPU bench path on the CPU: a single cut does not shard, so N GPUs
run N replicas and the job's time is the slowest rank's.  Two gloo ranks
check the aggregate the bench reports (max over ranks, whole-job units/s)
and that every rank takes the same collective steps."""
from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms, value = bench.whole_job(1_000_000, 10.0 + 5.0 * rank, world)
        bench.barrier(world)
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_replica_aggregate_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in procs)
    for rank, ms, value in got:
        assert ms == 15.0                       # the slowest rank's time
        assert value == 2 * 1_000_000 / 15e-3   # all ranks' units over that time


def test_single_rank_aggregate():
    import bench

    assert bench.whole_job(500, 2.0, 1) == (2.0, 500 / 2e-3)
