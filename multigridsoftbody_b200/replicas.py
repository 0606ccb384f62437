"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host side.

A single body does not shard (a domain split would need a halo exchange every
sweep), so N GPUs run N independent replicas.  A batch of bodies shards by
body: bodies are assigned to ranks by tet count (longest-processing-time
greedy), with no collective on the data path; only the timing reduction
(max over ranks) and an optional gather of results use the process group.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_bodies(tet_counts, world_size: int) -> list[list[int]]:
    """Greedy LPT assignment of bodies to ranks; deterministic (ties by body index)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(tet_counts)), key=lambda i: (-int(tet_counts[i]), i))
    heap = [(0, r) for r in range(world_size)]
    heapq.heapify(heap)
    out = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(tet_counts[i]), r))
    return [sorted(s) for s in out]


class BodyShard:
    """One rank's share of a batch of independent bodies: the body indices that
    `shard_bodies` assigns to this rank, and views of per-body inputs."""

    def __init__(self, tet_counts, world_size: int, rank: int):
        if not 0 <= rank < world_size:
            raise ValueError(f"rank {rank} outside world size {world_size}")
        self.num_bodies = len(tet_counts)
        self.bodies = shard_bodies(tet_counts, world_size)[rank]

    def take(self, per_body):
        """This rank's entries of a per-body list (None stays None)."""
        return None if per_body is None else [per_body[i] for i in self.bodies]

    def tool(self, tool):
        """Wrap a per-frame tool callback returning (a[n, 3], b[n, 3], r[n]) for all n bodies so that it
        returns this rank's rows, in the order of `bodies`."""
        idx = np.asarray(self.bodies, dtype=np.int64)

        def f(frame):
            a, b, r = tool(frame)
            return a[idx], b[idx], r[idx]

        return f


def max_over_ranks(values, dist=None):
    """Element-wise max of per-rank timings (the job's time is its slowest rank)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64)
    if dist is not None and dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if dist.get_backend() == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_throughput(frames_per_rank: int, world_size: int, max_ms: float) -> float:
    """Whole-job frames/s of independent replicas: all ranks' frames over the slowest rank's time."""
    return frames_per_rank * world_size / (max_ms / 1e3)


def sharded_throughput(frames: int, max_ms: float) -> float:
    """Frames/s of a batch sharded by body: a frame advances every body once, on whichever rank holds it,
    so the batch runs `frames` frames in the slowest rank's time."""
    return frames / (max_ms / 1e3)
