"""Sharding independent problems across ranks (one process per GPU).

Independent grids need no exchange while they step, so a multi-GPU batch is
a partition of the problems plus a gather of results at the end: each rank
builds a `Batch` of its own share and steps it; nothing crosses between GPUs
on the data path. The partition balances the cost of a share, cells x steps,
with the longest-processing-time rule (largest problem first, onto the rank
with the least cost so far; ties go to the lower rank), so every rank computes
the same partition from the same problem list without communicating.
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np


def problem_cost(p) -> float:
    """Cell-updates of a problem: interior cells x steps."""
    return float(p.interior_cells) * float(max(1, p.steps))


def partition_by_cost(costs: Sequence[float], world: int) -> List[List[int]]:
    """Indices of the problems each of `world` ranks takes. Deterministic;
    every index appears exactly once; within a share, indices ascend."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda q: (-float(costs[q]), q))
    load = [0.0] * world
    shares: List[List[int]] = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shares[r].append(q)
        load[r] += float(costs[q])
    return [sorted(s) for s in shares]


def shard_for_rank(problems: Sequence, rank: int, world: int) -> List[int]:
    """Indices of `problems` that rank `rank` of `world` steps."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return partition_by_cost([problem_cost(p) for p in problems], world)[rank]


def imbalance(costs: Sequence[float], shares: List[List[int]]) -> float:
    """Largest share cost over the mean share cost (1.0 = perfect)."""
    loads = np.array([sum(costs[q] for q in s) for s in shares], dtype=np.float64)
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0


def gather_results(local: Dict[int, np.ndarray], group=None, dst: int = 0):
    """Collect {problem index: array} from every rank on rank `dst` (over the
    process group's backend; returns the merged dict on `dst`, None
    elsewhere). A problem reported by two ranks is an error."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = [None] * world if rank == dst else None
    dist.gather_object(local, parts, dst=dst, group=group)
    if rank != dst:
        return None
    merged: Dict[int, np.ndarray] = {}
    for part in parts:
        for q, v in part.items():
            if q in merged:
                raise RuntimeError(f"problem {q} reported by two ranks")
            merged[q] = v
    return merged
