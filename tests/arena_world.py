"""A small dynamic world for the scene-cache tests (test helper), shaped like the reference's
incremental-rebuild tests (bench.rs:488-560): bodies whose worldline histories grow by a few
samples per snapshot (some with causal decision stamps), pieces keyed by the caller (as laser
pulses are), a volatile part made afresh every snapshot, a body that leaves, and a rebase that
shifts everything in lab time.

Samples are inertial: centre (t, x0 + v t), the boost tetrad of v, proper time t / gamma (the
standard Lorentz boost, e0 = gamma (1, v), e_i = (gamma v_i, delta_ij + (gamma - 1) v_i v_j / v^2)).
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

TRI_DTYPE = O.TRI_DTYPE
SAMPLE_DTYPE = O.SAMPLE_DTYPE


def boost_tetrad(v):
    v = np.asarray(v, np.float64)
    v2 = float(v @ v)
    g = 1.0 / np.sqrt(1.0 - v2)
    e = np.zeros((4, 4))
    e[0, 0] = g
    e[0, 1:] = g * v
    for i in range(3):
        e[i + 1, 0] = g * v[i]
        for j in range(3):
            e[i + 1, j + 1] = (1.0 if i == j else 0.0) + ((g - 1.0) * v[i] * v[j] / v2 if v2 > 0 else 0.0)
    return e, g


def inertial_samples(x0, v, t0, dt, n):
    e, g = boost_tetrad(v)
    s = np.zeros(n, SAMPLE_DTYPE)
    t = t0 + dt * np.arange(n)
    s["center"][:, 0] = t
    s["center"][:, 1:] = np.asarray(x0)[None, :] + np.outer(t, v)
    s["tetrad"][:] = e.astype(np.float32)[None]
    s["proper_time"] = (t / g).astype(np.float32)
    return s


class World:
    """Bodies, pieces and a volatile part; snapshot(k) says what the k-th snapshot holds."""

    def __init__(self, mesh_tube, simplices, seed: int = 3, n_bodies: int = 6, base: int = 6):
        rng = np.random.default_rng(seed)
        self.base = base
        self.vertices = (mesh_tube.vertices * np.float32(3.0)).astype(np.float32)  # larger bodies: more hits
        self.triangles = mesh_tube.triangles
        self.bodies = []
        for b in range(n_bodies):
            x0 = rng.uniform(-6, 6, 3)
            v = rng.uniform(-0.5, 0.5, 3)
            dt = float(rng.choice([0.3, 0.45, 1.7]))   # several samples per 1.0 of lab time, or fewer
            decided = b % 2 == 1
            self.bodies.append(dict(x0=x0, v=v, dt=dt, t0=-12.0, decided=decided, material=int(b % 6)))
        self.boxes, self.geoms, self.attrs = simplices
        self.shift = 0.0

    def tube_of(self, b: int, k: int):
        body = self.bodies[b]
        n = self.base + 3 * k + b  # the history grows by three samples per snapshot
        s = inertial_samples(body["x0"], body["v"], body["t0"], body["dt"], n)
        s["center"][:, 0] += np.float32(self.shift)
        dec = (s["center"][:, 0] - np.float32(0.5)).astype(np.float32) if body["decided"] else None
        return s, dec

    def pieces(self, k: int):
        """(index, key, slice of simplices): piece i of the pulse; the last one changes every snapshot."""
        out = []
        n = min(4, 1 + k)
        for i in range(n):
            last = i == n - 1
            lo = 40 * i
            hi = lo + (20 + k if last else 30)
            key = [i, lo, hi]  # what the piece is made from (not moved by a rebase)
            out.append((i, key, slice(lo, hi)))
        return out

    def volatile(self, k: int):
        lo = 200 + 7 * k
        return slice(lo, lo + 60)

    def bodies_at(self, k: int):
        """Body 2 leaves the world at snapshot 4."""
        return [b for b in range(len(self.bodies)) if not (b == 2 and k >= 4)]

    def scratch(self, k: int):
        """Snapshot k's simplices made at once (whole tubes, then pieces, then the volatile part):
        boxes, hot and cold records in build order."""
        parts = []
        for b in self.bodies_at(k):
            s, dec = self.tube_of(b, k)
            parts.append(O.tube_simplices(self.vertices, self.triangles, s, self.bodies[b]["material"], dec))
        for _, _, sl in self.pieces(k):
            parts.append((self.boxes[sl], self.geoms[sl], self.attrs[sl]))
        sl = self.volatile(k)
        parts.append((self.boxes[sl], self.geoms[sl], self.attrs[sl]))
        return tuple(np.concatenate([p[i] for p in parts]) for i in range(3))

    def drive(self, k: int, arena_begin, arena_tube, arena_piece, arena_finish):
        """One snapshot through the four scene-cache calls (engine or oracle)."""
        arena_begin()
        for b in self.bodies_at(k):
            s, dec = self.tube_of(b, k)
            arena_tube((0, 0, 100 + b), s, dec, self.bodies[b]["material"])
        for i, key, sl in self.pieces(k):
            arena_piece((2, 1, 7), i, key, self.boxes[sl], self.geoms[sl], self.attrs[sl])
        sl = self.volatile(k)
        return arena_finish(self.boxes[sl], self.geoms[sl], self.attrs[sl])


def record_rows(geoms, attrs):
    return sorted(geoms[i].tobytes() + attrs[i].tobytes() for i in range(len(geoms)))


def in_tree(nodes, geoms, attrs):
    """The records reachable from the root (Bvh4D::in_tree, bvh4d.rs:226-250), as sorted bytes."""
    out = []
    if len(nodes) == 0:
        return out
    n0 = nodes[0]
    if n0["count"] == 0 and n0["left"] == 0 and n0["right_or_first"] == 0 and (n0["min"] > n0["max"]).any():
        return out
    stack = [0]
    seen = set()
    while stack:
        i = stack.pop()
        assert i not in seen, "node reached twice"
        seen.add(i)
        nd = nodes[i]
        if nd["count"] > 0:
            a = int(nd["right_or_first"])
            for p in range(a, a + int(nd["count"])):
                out.append(geoms[p].tobytes() + attrs[p].tobytes())
        else:
            stack += [int(nd["left"]), int(nd["right_or_first"])]
    return sorted(out)
