"""The multi-GPU host logic on CPU: two gloo ranks on 127.0.0.1 shard the observers as bench.py does
(one seeded stream per rank, no observer on two ranks) and reduce the timing as the max over ranks.
The render path itself has no collective, so nothing else crosses ranks."""
import datetime
import os
import socket

import pytest

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        from specrel_b200 import shard
        raps = shard.observer_rapidities(5, rank, 6, first=(0.1, 0.2, 0.3))
        gathered = [None] * WORLD
        dist.all_gather_object(gathered, raps)
        slowest = shard.max_over_ranks(1.5 + rank, dist)
        dist.barrier()
        q.put((rank, gathered, slowest, shard.total_rays(1000, WORLD)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_observers_and_reduce_the_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=180) for _ in range(WORLD))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    (_, g0, m0, n0), (_, g1, m1, n1) = results
    assert g0 == g1
    r0, r1 = g0
    assert r0[0] == (0.1, 0.2, 0.3)
    assert not set(r0) & set(r1)
    assert all(sum(x * x for x in phi) <= 4.0 + 1e-12 for phi in r0 + r1)
    assert m0 == m1 == 2.5
    assert n0 == n1 == 2000


class _BandEngine:
    """Stands in for the engine's sr_adjoint_rows: each loss-level row r adds (r + 1) * (1, 2, ..., 10)
    to the ten results, so the reduced sum checks that the bands cover every row exactly once."""

    def adjoint(self, idx, u, cam, target, level, rows=None):
        import types
        r0, r1 = rows
        w = sum(r + 1 for r in range(r0, r1))
        return types.SimpleNamespace(loss=1.0 * w, grad=[(k + 2.0) * w for k in range(7)], primal_mismatch=9.0 * w,
                                     star_terms=10.0 * w)


def _adjoint_worker(rank, port, q):
    import types
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        from specrel_b200 import shard
        u = types.SimpleNamespace(size=(160, 101))
        out = shard.adjoint_over_ranks(_BandEngine(), 0, u, None, 0, level=2, dist=dist)
        q.put((rank, shard.row_band(shard.loss_rows(101, 2), rank, WORLD), [float(x) for x in out]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_the_gradient_rows_and_sum_them():
    """The sharded gradient (the one collective of the path): two gloo ranks take contiguous
    bands of the loss level's rows and one all-reduce gives both the whole frame's results."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_adjoint_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=180) for _ in range(WORLD))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    (_, b0, o0), (_, b1, o1) = results
    rows = 26  # 101 -> 51 -> 26
    assert b0 == (0, 13) and b1 == (13, 26)
    w = sum(r + 1 for r in range(rows))
    assert o0 == o1 == [1.0 * w] + [(k + 2.0) * w for k in range(7)] + [9.0 * w, 10.0 * w]


def test_single_process_needs_no_group():
    from specrel_b200 import shard
    assert shard.max_over_ranks(3.0) == 3.0
    a = shard.observer_rapidities(5, 1, 4)
    assert a == shard.observer_rapidities(5, 1, 4)
    assert a != shard.observer_rapidities(5, 0, 4)


def _c_reduce_worker(rank, port, q):
    """The C-level path a non-Python host takes: sr_adjoint_band for the rank's rows, then
    sr_adjoint_reduce with the caller's sum (here gloo's all-reduce behind a C function pointer)."""
    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        from specrel_b200 import _lib as L
        from specrel_b200 import shard
        lib = L.lib()
        bands = []
        for level in (0, 3, 6):
            r0, r1 = C.c_uint32(), C.c_uint32()
            assert lib.sr_adjoint_band(800, level, rank, WORLD, C.byref(r0), C.byref(r1)) == L.SR_OK
            bands.append((r0.value, r1.value, shard.row_band(shard.loss_rows(800, level), rank, WORLD)))
        calls = []

        @L.SUM_F64_FN
        def gloo_sum(values, count, user):
            t = torch.tensor(np.ctypeslib.as_array(values, shape=(count,)).copy())
            dist.all_reduce(t)
            for k in range(count):
                values[k] = float(t[k])
            calls.append(count)
            return 0

        part = L.AdjointResult()
        part.loss = 1.5 + rank
        for k in range(7):
            part.grad[k] = (rank + 1) * (k - 3) * 0.25
        part.primal_mismatch = 0.0
        part.star_terms = 100.0 * (rank + 1)
        assert lib.sr_adjoint_reduce(C.byref(part), gloo_sum, None) == L.SR_OK
        q.put((rank, bands, part.loss, list(part.grad), part.primal_mismatch, part.star_terms, calls))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_the_gradient_through_the_c_abi():
    """Two gloo ranks: the library's row bands equal the Python harness's, and sr_adjoint_reduce
    sums the ten doubles of SrAdjointResult through the caller's sum function."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_c_reduce_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=180) for _ in range(WORLD))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank, bands, loss, grad, pm, stars, calls in results:
        for r0, r1, ref in bands:
            assert (r0, r1) == ref
        assert loss == 1.5 + 2.5
        assert grad == [3 * (k - 3) * 0.25 for k in range(7)]
        assert pm == 0.0 and stars == 300.0
        assert calls == [10]
