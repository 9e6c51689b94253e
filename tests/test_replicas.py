"""Multi-GPU plumbing of bench.py on the CPU: world size 2 over gloo (127.0.0.1).

The path shards as replicas: every rank runs its own cloud (seeded by its rank) with no
data-path collective; the bench's only collectives are a barrier around the timed region and a
max over ranks of the timings.  Here two ranks check that the max reduction and the barrier
behave, and that the replicas' clouds differ."""
import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import workloads
        bench.barrier(world)
        got = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        cloud = workloads.jittered_lattice(6, rank)
        bench.barrier(world)
        q.put((rank, got, float(cloud.sum())))
    finally:
        dist.destroy_process_group()


def test_two_replica_ranks_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [15.0, 15.0]  # the max over ranks on every rank
    assert res[0][2] != res[1][2]  # independent clouds
