"""Sharding over ranks (one process per GPU).

The render path has no exchange between observers: each rank renders its own batch of observers
on its own GPU, against its own replica of the scene, and only the timing is reduced (max over
ranks). The gradient of one observer's image loss is sharded by rows of the loss level: each rank
evaluates its band (sr_adjoint_rows) and one all-reduce of ten doubles (loss, gradient, primal
mismatches, star terms) gives every rank the whole. These helpers hold that host-side logic so it
can be tested with the gloo backend on CPU.
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


def row_band(rows: int, rank: int, world: int) -> tuple[int, int]:
    """Rank `rank`'s band of `rows` rows: contiguous, the sizes differing by at most one."""
    return rows * rank // world, rows * (rank + 1) // world


def loss_rows(height: int, level: int) -> int:
    """Rows of the loss level: `level` halvings of the frame's height, rounding up."""
    for _ in range(level):
        height = (height + 1) // 2
    return height


def adjoint_over_ranks(engine, idx: int, u, cam, target_hdr_ptr: int, level: int = 0, dist=None,
                       device: str = "cpu"):
    """One observer's loss and gradient, its rows sharded over the ranks of the default process
    group: (loss, grad[7], primal mismatches, star terms) as a numpy array, the same on every rank.
    Every rank holds the scene and the target; a rank whose band is empty adds nothing."""
    import torch
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    r0, r1 = row_band(loss_rows(int(u.size[1]), level), rank, world)
    part = np.zeros(10)
    if r1 > r0:
        r = engine.adjoint(idx, u, cam, target_hdr_ptr, level, rows=(r0, r1))
        part[0] = r.loss
        part[1:8] = [r.grad[k] for k in range(7)]
        part[8] = r.primal_mismatch
        part[9] = r.star_terms
    if world == 1:
        return part
    t = torch.tensor(part, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()
