"""Energy points sharded over GPUs (one process per GPU), results gathered on every rank.

Every (energy, pair, L) is independent (the reference's driver loops over energies,
driver.py:872-1152, and over ejected energies in ionization.py:526-608), so the only exchange is
the final gather of the results: no operand or tile crosses GPUs. Points are assigned largest
first to the least-loaded rank (cost = N^2 x pairs x transitions, the dense-equivalent work of a
point), which is deterministic, so every rank derives the same assignment without communication.
The gather goes through ``torch.distributed.all_gather_object`` (host objects: one small list of
I_L per point), on whatever process group the caller set up (NCCL on the GPUs, gloo on hosts).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np

__all__ = ["point_cost", "partition_points", "radial_ME_all_L_sweep_distributed"]


def point_cost(pt: dict) -> float:
    """Dense-equivalent work of one energy point: N^2 x pairs x transitions."""
    N = len(pt["grid"].r)
    n_t = len(pt["bound_i"]) if isinstance(pt["bound_i"], (list, tuple)) else 1
    return float(N) * N * len(pt["pairs"]) * n_t


def partition_points(costs: Sequence[float], world_size: int) -> List[List[int]]:
    """Longest-processing-time assignment: points by decreasing cost (ties by index) to the rank
    with the least load so far (ties by rank). Each rank's list is returned in ascending order."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = np.zeros(world_size)
    parts: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = int(np.argmin(load))  # first minimum: lowest rank among ties
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def radial_ME_all_L_sweep_distributed(points: Sequence[dict], L_max: int, group=None,
                                      compute: Optional[Callable] = None, **options):
    """``radial_ME_all_L_sweep`` over the ranks of ``group``: each rank evaluates its share of the
    points (on its own GPU) and every rank returns the results of all points, in input order.
    ``compute(points, L_max, **options)`` defaults to ``radial_ME_all_L_sweep``."""
    import torch.distributed as dist
    if compute is None:
        from .dwba_matrix_elements import radial_ME_all_L_sweep as compute
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = partition_points([point_cost(p) for p in points], world)
    mine = parts[rank]
    local = compute([points[i] for i in mine], L_max, **options) if mine else []
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (mine, local), group=group)
    out: list = [None] * len(points)
    for idx, res in gathered:
        for i, r in zip(idx, res):
            out[i] = r
    return out
