"""Scene-parallel placement for the batched and served forms on several GPUs.

Scenes are independent, so N GPUs run N engines with no collective on the data path: each
rank takes a share of the scenes (longest-processing-time greedy on particle counts,
deterministic so every rank computes the same assignment without talking), and the only
cross-rank traffic is the timing reduction of the benchmark (max over ranks).
"""
from __future__ import annotations


def assign_scenes(sizes, world: int) -> list:
    """Indices of the scenes each rank steps: scenes in descending size (ties by index)
    go to the least-loaded rank (ties by rank). Returns `world` ascending index lists."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out = [[] for _ in range(world)]
    for q in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(q)
        load[r] += int(sizes[q])
    return [sorted(x) for x in out]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest of every rank's `value` (the slowest rank's time); `value` itself on
    one rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
