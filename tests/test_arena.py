"""The scene cache over an arena (SceneCache, dynamic/scene_cache.rs; Bvh4D's arena edits,
bvh4d.rs:168-215, 583-644) in the CPU oracle, held to the properties the reference's own tests
check (bench.rs:488-560): an incremental snapshot holds the same simplices as a rebuild from
scratch and its tree finds the same hits; most of a growing world is reused; a rebase rebuilds
everything and compacts the arena; the free room stays bounded. The engine's device arena is held
to this oracle byte for byte in test_arena_gpu.py."""
import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O

import arena_world as W


@pytest.fixture(scope="module")
def inputs():
    sc = sr.synth_scene(1, 1, n_bodies=4, steps=8)
    boxes, geoms, attrs, p = sc.build_inputs()
    return sc.tubes()[0], (boxes, geoms, attrs), p.materials


def drive(w, A, k):
    return w.drive(k, A.begin, lambda part, s, d, m: A.tube(part, w.vertices, w.triangles, s, m, d), A.piece, A.finish)


def hits(nodes, geoms, attrs, mats):
    """The past light cone of an observer at the origin, looking four ways: (slot, lambda, rgb)."""
    scene = O.Scene.from_packed(nodes, geoms, attrs, mats, np.zeros(4, np.float32), 0)
    out = []
    for yaw in (0.0, 90.0, 180.0, 270.0):
        cam = O.make_camera(pos=(0.0, 0.0, 0.0, 0.0), fov_deg=100.0, yaw=yaw)
        r = O.render(scene, cam, O.make_config(96, 64), threads=4)
        out.append((r.slot, r.lam, r.rgb))
    return tuple(np.concatenate([o[i] for o in out]) for i in range(3))


def test_incremental_snapshot_matches_a_rebuild_from_scratch(inputs):
    tube, simplices, mats = inputs
    w = W.World(tube, simplices)
    A = O.Arena()
    stats = [drive(w, A, k) for k in range(10)]
    nodes, g, a = A.arrays()
    b, gs, as_ = w.scratch(9)
    assert W.in_tree(nodes, g, a) == W.record_rows(gs, as_)
    last = stats[-1]
    assert last["simplices_built"] * 4 < last["simplices_reused"], last
    assert all(s["compacted"] == 0 for s in stats)
    # One tree over everything (the volatile part of a fresh cache) finds the same hits.
    S = O.Arena()
    S.begin()
    S.finish(b, gs, as_)
    (sa, la, ca), (ss, ls, cs) = hits(nodes, g, a, mats), hits(*S.arrays(), mats)
    assert (sa >= 0).sum() > 2000
    assert ((sa >= 0) == (ss >= 0)).all() and (la == ls).all() and (ca == cs).all()


def test_rebase_rebuilds_everything_and_compacts(inputs):
    tube, simplices, mats = inputs
    w = W.World(tube, simplices, n_bodies=12, base=60)
    A = O.Arena()
    for k in range(3):
        drive(w, A, k)
    w.shift = -7.25
    stats = [drive(w, A, 3) for _ in range(3)]
    # Every tube chunk is rebuilt; the pulse's pieces (not moved) are kept and moved together.
    assert stats[0]["chunks_reused"] == 2 and stats[0]["simplices_reused"] == 60, stats[0]
    assert stats[0]["compacted"] == 1, stats[0]
    assert stats[1]["simplices_built"] < stats[1]["simplices_reused"] / 20
    nodes, g, a = A.arrays()
    b, gs, as_ = w.scratch(3)
    live = W.in_tree(nodes, g, a)
    assert live == W.record_rows(gs, as_)
    assert stats[-1]["arena_simplices"] < 2 * len(live) + (1 << 15)


def test_space_first_fit_and_merging():
    """Space (scene_cache.rs:72-115) through the arena: dropped chunks leave room that the next
    chunks fill first, and room freed at the end shrinks the arena."""
    sc = sr.synth_scene(1, 1, n_bodies=4, steps=8)
    boxes, geoms, attrs, _ = sc.build_inputs()
    A = O.Arena()
    A.begin()
    for i in range(4):
        A.piece((2, 0, 1), i, [i], boxes[40 * i:40 * i + 30], geoms[40 * i:40 * i + 30], attrs[40 * i:40 * i + 30])
    s = A.finish()
    assert s["arena_simplices"] == 120 and s["chunks_built"] == 4
    A.begin()  # pieces 1 and 3 dropped, piece 4 made: it goes into piece 1's room
    for i in (0, 2, 4):
        A.piece((2, 0, 1), i, [i], boxes[40 * i:40 * i + 30], geoms[40 * i:40 * i + 30], attrs[40 * i:40 * i + 30])
    s = A.finish()
    assert s["chunks_reused"] == 2 and s["chunks_built"] == 1
    assert s["arena_simplices"] == 90  # piece 3's room at the end is given back
    nodes, g, a = A.arrays()
    assert W.record_rows(g[30:60], a[30:60]) == W.record_rows(geoms[160:190], attrs[160:190])  # leaf order


@pytest.mark.parametrize("n,quant", [(2, 0.0), (3, 0.0), (57, 0.0), (1430, 0.0), (400, 2.0), (900, 0.5)])
def test_top_tree_equals_the_restatement(n, quant):
    """The engine's top_tree (sorted indices, merge sorts, the last sort skipped without ties)
    against the oracle's plain restatement; `quant` snaps centres to a grid so that many items tie
    on one or more axes (bodies at rest, identical boxes)."""
    rng = np.random.default_rng(n)
    c = rng.uniform(-20, 20, (n, 4)).astype(np.float32)
    if quant:
        c = (np.round(c / quant) * quant).astype(np.float32)
        c[::7, 1:] = c[0, 1:]  # a body at rest: many chunks with one spatial centre
        c[5::11] = c[5]        # identical boxes
    e = rng.uniform(0.05, 2.0, (n, 4)).astype(np.float32)
    if quant:
        e[5::11] = e[5]
    boxes = np.concatenate([c - e, c + e], axis=1).astype(np.float32)
    roots = rng.integers(1, 1 << 20, n).astype(np.uint32)
    weights = rng.integers(1, 300, n).astype(np.float32)
    base = 1000
    ref = O.top_tree(boxes, roots, weights, base)
    got, depth = sr.top_tree(boxes, roots, weights, base, depths=np.full(n, 3, np.uint32))
    assert got.tobytes() == ref.tobytes()
    assert depth >= 4


def test_dirty_ranges_patch_a_copy_into_the_arena():
    """PackedSceneGpuData::update (gpu.rs:296-315): a copy of the arrays patched with each edit's
    dirty ranges, when it holds the edit before of the same layout (else copied afresh), equals the
    arrays; most snapshots are patched (bench.rs:488-510)."""
    sc = sr.synth_scene(1, 1, n_bodies=4, steps=8)
    boxes, geoms, attrs, p = sc.build_inputs()
    w = W.World(sc.tubes()[0], (boxes, geoms, attrs))
    A = O.Arena()
    copy, version, patched = None, None, 0
    for k in range(10):
        drive(w, A, k)
        lay, ed, nr, pr = A.dirty()
        nodes, g, a = A.arrays()
        if version is not None and version == (lay, ed - 1):
            cn, cg, ca = copy
            cn = np.concatenate([cn, np.zeros(max(0, len(nodes) - len(cn)), cn.dtype)])
            cg = np.concatenate([cg, np.zeros(max(0, len(g) - len(cg)), cg.dtype)])
            ca = np.concatenate([ca, np.zeros(max(0, len(a) - len(ca)), ca.dtype)])
            for s, e in nr:
                cn[s:e] = nodes[s:e]
            for s, e in pr:
                cg[s:e] = g[s:e]
                ca[s:e] = a[s:e]
            copy = (cn, cg, ca)
            patched += 1
        else:
            copy = (nodes.copy(), g.copy(), a.copy())
        version = (lay, ed)
        assert all(x.tobytes() == y.tobytes() for x, y in zip(copy, (nodes, g, a))), k
    assert patched == 9


def test_single_chunk_root_and_nothing():
    """One chunk: node 0 is a copy of its root (scene_cache.rs:328); nothing: node 0 over nothing."""
    sc = sr.synth_scene(1, 1, n_bodies=4, steps=8)
    boxes, geoms, attrs, _ = sc.build_inputs()
    A = O.Arena()
    A.begin()
    A.piece((2, 0, 1), 0, [0], boxes[:25], geoms[:25], attrs[:25])
    A.finish()
    nodes, g, a = A.arrays()
    assert nodes[0].tobytes() == nodes[1].tobytes()  # the chunk's root went to node 1
    assert W.in_tree(nodes, g, a) == W.record_rows(geoms[:25], attrs[:25])
    A.begin()
    A.finish()
    nodes, g, a = A.arrays()
    assert nodes[0]["count"] == 0 and nodes[0]["left"] == 0 and nodes[0]["right_or_first"] == 0
    assert (nodes[0]["min"] > nodes[0]["max"]).all()
    assert W.in_tree(nodes, g, a) == []


def test_validation_takes_the_reference_arena_arrays():
    """The arrays the reference's dynamic flow uploads (an arena's, free room included) pass the
    upload's checks; a root over nothing (an empty arena) is an empty tree; a real cycle is refused."""
    sc = sr.synth_scene(1, 1, n_bodies=4, steps=8)
    boxes, geoms, attrs, p = sc.build_inputs()
    w = W.World(sc.tubes()[0], (boxes, geoms, attrs))
    A = O.Arena()
    for k in range(5):
        drive(w, A, k)
    nodes, g, a = A.arrays()
    st, depth, msg = sr.validate(sr.PackedScene(nodes, g, a, p.materials, np.zeros(4, np.float32), 0))
    assert st == 0 and depth > 3, msg
    E = O.Arena()
    E.begin()
    E.finish()
    en, eg, ea = E.arrays()
    st, depth, msg = sr.validate(sr.PackedScene(en, eg, ea, p.materials, np.zeros(4, np.float32), 0))
    assert st == 0 and depth == 1, msg
    bad = nodes.copy()
    bad[0]["min"] = bad[0]["max"]  # a real box: node 0 linking to itself is now a cycle
    bad[0]["count"] = 0
    bad[0]["left"] = 0
    bad[0]["right_or_first"] = 0
    st, _, msg = sr.validate(sr.PackedScene(bad, g, a, p.materials, np.zeros(4, np.float32), 0))
    assert st != 0 and "twice" in msg


def test_top_tree_needs_two_items():
    with pytest.raises(sr.SrError):
        sr.top_tree(np.zeros((1, 8), np.float32), np.zeros(1, np.uint32), np.ones(1, np.float32), 0)
