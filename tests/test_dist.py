"""Multi-GPU plumbing of bench.py on CPU: two gloo ranks.

The batched workload shards by problem (each rank solves its own batch, no
data-path collective); the only collectives are a barrier and the max over
ranks of the timed interval.  Checked here without a GPU: every rank draws a
different, reproducible batch, and allmax returns the slowest rank's time on
every rank.
"""
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


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        probs = bench.shard_problems(rank)
        seeds = [p.seed for p in probs]
        slowest = bench.allmax(world, 1.0 + rank)  # rank r "took" 1 + r seconds
        bench.barrier(world)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        out[rank] = (slowest, len(probs), gathered)
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_timing():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        slowest, n, gathered = out[r]
        assert slowest == float(world)  # max over ranks
        assert n == 512
        assert not set(gathered[0]) & set(gathered[1])  # disjoint problems per rank
    # Reproducible: rank 1's batch is the same when drawn again here.
    import bench
    assert [p.seed for p in bench.shard_problems(1)] == out[1][2][1]
