"""Multi-rank host logic on CPU (gloo, world size 2): body sharding agreement and
the max-over-ranks timing reduction used by bench.py."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from multigridsoftbody_b200.replicas import job_throughput, max_over_ranks, shard_bodies


def test_shard_bodies_balanced_and_complete():
    import numpy as np
    rng = np.random.default_rng(11)
    ns = rng.integers(2, 9, size=256)
    tets = [6 * n * 10 * n * n for n in ns]
    for world in (1, 2, 4, 8):
        shards = shard_bodies(tets, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(256))
        loads = [sum(tets[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(tets)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tets = [100, 900, 400, 400, 300, 50, 700]
        mine = shard_bodies(tets, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        ms = max_over_ranks([10.0 + rank, 5.0 * (rank + 1)], dist)
        q.put((rank, gathered, ms))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, gathered, ms in res:
        assert sorted(i for s in gathered for i in s) == list(range(7))
        assert gathered == res[0][1]           # every rank computed the same assignment
        assert ms == [11.0, 10.0]              # element-wise max over ranks
    assert job_throughput(100, 2, 1000.0) == pytest.approx(200.0)
