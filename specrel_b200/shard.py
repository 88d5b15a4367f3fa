"""Sharding observers over ranks (one process per GPU).

The render path has no exchange between observers: each rank renders its own batch of observers
on its own GPU, against its own replica of the scene, and only the timing is reduced (max over
ranks). These helpers hold that host-side logic so it can be tested with the gloo backend on CPU.
"""
from __future__ import annotations

import numpy as np


def observer_rapidities(seed: int, rank: int, n: int, first=None) -> list[tuple[float, float, float]]:
    """Rapidities of rank `rank`'s `n` observers: seeded draws uniform in the ball |phi| <= 2, one
    stream per rank (so ranks never share an observer); rank 0's first observer is `first` when
    given (the workload's own observer)."""
    rng = np.random.default_rng(seed * 7919 + rank)
    out = []
    for i in range(n):
        if rank == 0 and i == 0 and first is not None:
            out.append(tuple(float(x) for x in first))
            continue
        while True:
            v = rng.uniform(-1.0, 1.0, 3)
            if v @ v < 1.0:
                break
        out.append(tuple(float(2.0 * x) for x in v))
    return out


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    """The maximum of `x` over all ranks of the default process group (x itself without one)."""
    if dist is None or not dist.is_initialized():
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def total_rays(rays_per_rank: int, world: int) -> int:
    """Weak scaling: every rank renders the same number of rays, the job renders world times that."""
    return rays_per_rank * world
