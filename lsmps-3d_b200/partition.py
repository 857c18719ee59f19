"""Partition of independent particle boxes over GPUs (one process per GPU).

Boxes share nothing, so a batch shards with no data-path collective: each
rank steps its own boxes (as one merged batch on its GPU) and the only
communication is the host-side reduction of the timing and the particle
count.  Boxes are assigned by the longest-processing-time rule: in
decreasing order of fluid count, each box goes to the rank with the least
load so far (ties to the lower rank), which keeps the largest rank within
4/3 of the optimum.
"""

from __future__ import annotations


def partition_boxes(sizes: list[int], world: int) -> list[list[int]]:
    """Box indices per rank (each list ascending), balanced by `sizes`."""
    if world < 1:
        raise ValueError("world must be at least 1")
    loads = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for b in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(b)
        loads[r] += int(sizes[b])
    return [sorted(p) for p in parts]


def reduce_rank_results(world: int, particles: int, ms: float, device=None) -> tuple[int, float]:
    """The whole job's particle count (sum over ranks) and time (max over
    ranks) through torch.distributed (any backend), or the rank's own
    values for a single process."""
    if world <= 1:
        return particles, ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(particles)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    m = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return int(t.item()), float(m.item())
