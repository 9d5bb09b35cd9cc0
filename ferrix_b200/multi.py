"""Multi-GPU plumbing for independent decks (one process per GPU).

A single deck is not sharded (its matrix fits one GPU many times over); many
independent decks are partitioned across the ranks by device-memory footprint,
with no collective on the data path. The only collectives are the timing
reduction (max over ranks) and barriers around the timed region.
"""
from __future__ import annotations

from typing import List, Sequence


def partition_by_footprint(sizes: Sequence[float], world: int) -> List[List[int]]:
    """Deterministic greedy partition (largest first onto the least-loaded rank,
    ties to the lower rank): every index lands on exactly one rank, and every
    rank computes the same partition from the same sizes."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-float(sizes[i]), i))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(sizes[i])
    for p in parts:
        p.sort()
    return parts


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
