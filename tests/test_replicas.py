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


class _FakeMesh:
    def __init__(self, tets):
        self.num_tets = tets
        self.num_verts = tets // 4


def _batch_worker(rank, world, port, q):
    """bench.py's sharded batch path on a fake solver: the rank's bodies, its tool rows, one frame per step."""
    import numpy as np
    import torch.distributed as dist

    import bench
    from multigridsoftbody_b200.replicas import max_over_ranks, sharded_throughput

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(11)
        ns = rng.integers(2, 9, size=256)
        meshes = [_FakeMesh(6 * 10 * int(n) ** 3) for n in ns]
        params = [("params", i) for i in range(256)]
        fixeds = [("fixed", i) for i in range(256)]
        mats = [("mat", i) for i in range(256)]

        def tool(f):   # body i's capsule: a = (i, f, 0), b = (i, f, 1), r = i
            a = np.stack([np.arange(256.0), np.full(256, float(f)), np.zeros(256)], 1)
            return a, a + [0.0, 0.0, 1.0], np.arange(256.0)

        m, p, fx, tl, mt, shard = bench.shard_workload(meshes, params, fixeds, tool, mats, world, rank)
        assert shard is not None and [x[1] for x in p] == shard.bodies == [x[1] for x in fx] == [x[1] for x in mt]
        stepped = []
        for f in range(5):   # the fake solver steps each of its bodies with its own tool row
            a, b, r = tl(f)
            for k, body in enumerate(shard.bodies):
                assert a[k, 0] == body and a[k, 1] == f and r[k] == body and b[k, 2] == 1.0
                stepped.append((body, f))
        gathered = [None] * world
        dist.all_gather_object(gathered, stepped)
        ms = max_over_ranks([100.0 * (rank + 1)], dist)[0]
        q.put((rank, gathered, ms, sharded_throughput(5, ms), sum(mm.num_tets for mm in m)))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_two_rank_gloo():
    """Every body of the 256-body batch is stepped exactly once per frame, on exactly one rank, with its
    own tool pose; the batch's frames/s comes from the slowest rank."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    steps = sorted(s for x in res[0][1] for s in x)
    assert steps == sorted((b, f) for b in range(256) for f in range(5))
    for rank, gathered, ms, fps, tets in res:
        assert ms == 200.0 and fps == pytest.approx(25.0)   # 5 frames in the slower rank's 200 ms
    loads = [r[4] for r in res]
    assert abs(loads[0] - loads[1]) <= 6 * 10 * 8 ** 3


def test_single_body_is_replicated():
    import bench
    m = [_FakeMesh(100)]
    out = bench.shard_workload(m, ["p"], ["f"], None, None, 4, 3)
    assert out[0] is m and out[-1] is None
