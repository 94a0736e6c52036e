"""Scene sharding across GPUs (one process per GPU, no data-path collective).

Acoustic scenes are independent (NAGA runs one ``simulation_engine`` per
scene, ``detail/simulation_engine.cuh``), so a multi-GPU job partitions its
scene set: each rank builds, steps and observes only its own scenes, and the
ranks meet only to agree on timing (max over ranks) and to add up the work
done. These helpers hold that host-side logic so it can run -- and be tested
-- with any ``torch.distributed`` backend (``nccl`` on GPUs, ``gloo`` on CPU).
"""
from __future__ import annotations

import heapq
from typing import Sequence


def partition_by_size(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Size-balanced greedy partition (longest processing time first).

    Scenes are taken in decreasing size (ties by index) and each goes to the
    rank with the least assigned nodes so far (ties by rank). Every rank
    computes the same partition from the same sizes. Returns, per rank, the
    scene indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda t: (-int(sizes[t]), t)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(o) for o in out]


def shard(sizes: Sequence[int], rank: int, world: int) -> list[int]:
    """The scene indices rank `rank` of `world` owns."""
    return partition_by_size(sizes, world)[rank]


class Router:
    """Online placement of serving requests: each request goes to the rank
    with the fewest outstanding node-steps (ties by rank). Deterministic, so
    every rank can run the same router on the same request stream and know
    which requests are its own without a message."""

    def __init__(self, world: int):
        if world < 1:
            raise ValueError("world must be >= 1")
        self.load = [0] * world

    def place(self, nodes: int, steps: int) -> int:
        r = min(range(len(self.load)), key=lambda t: (self.load[t], t))
        self.load[r] += int(nodes) * int(steps)
        return r

    def done(self, rank: int, nodes: int, steps: int) -> None:
        self.load[rank] -= int(nodes) * int(steps)


def _reduce(value: float, dist, op_name: str, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The slowest rank's time: the job's time."""
    return _reduce(value, dist, "MAX", device)


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """Work done by all ranks (node updates, scenes)."""
    return _reduce(value, dist, "SUM", device)
