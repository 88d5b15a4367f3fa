"""The engine's scene cache over its device arena (sr_arena_*) against the oracle's (test_arena.py
holds the oracle to the properties the reference's own tests check): after every snapshot the node
array and the hot and cold records, free room included, equal the oracle arena's byte for byte, the
CacheStats agree, and frames rendered from the arena equal frames rendered from the same arrays
uploaded with sr_upload_scene (the reference's path: the host arena patched into the GPU copy)."""
import time

import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O

import arena_world as W

pytestmark = pytest.mark.gpu

IDX, UPLOADED = 31, 32


@pytest.fixture(scope="module")
def inputs():
    sc = sr.synth_scene(1, 1, n_bodies=4, steps=8)
    boxes, geoms, attrs, p = sc.build_inputs()
    return sc, sc.tubes()[0], (boxes, geoms, attrs), p


def engine_drive(eng, w, k, rest, idx=IDX):
    return w.drive(k, lambda: eng.arena_begin(idx),
                   lambda part, s, d, m: eng.arena_tube(idx, part, sr.TubeData(w.vertices, w.triangles, s, m, d)),
                   lambda part, i, key, b, g, a: eng.arena_piece(idx, part, i, key, b, g, a),
                   lambda b, g, a: eng.arena_finish(idx, rest, b, g, a))


def oracle_drive(A, w, k):
    return w.drive(k, A.begin, lambda part, s, d, m: A.tube(part, w.vertices, w.triangles, s, m, d), A.piece,
                   A.finish)


def assert_same_arena(eng, A, idx=IDX):
    nodes, order = eng.tree(idx)
    g, a = eng.records(idx)
    on, og, oa = A.arrays()
    assert len(nodes) == len(on) and len(g) == len(og)
    assert nodes.tobytes() == on.tobytes()
    assert g.tobytes() == og.tobytes() and a.tobytes() == oa.tobytes()
    assert (order == np.arange(len(g))).all()  # hit ids are arena slots
    return on, og, oa


def assert_same_frames(eng, arrays, p, yaw, idx=IDX):
    nodes, geoms, attrs = arrays
    up = sr.PackedScene(nodes, geoms, attrs, p.materials, np.zeros(4, np.float32), 0, tuple(p.light_pos),
                        anchor=p.anchor)
    eng.upload(UPLOADED, up)
    u = sr.uniforms(sr.camera(fov_deg=100.0, yaw=yaw), 320, 200, 0, 1, 0, num_nodes=len(nodes),
                    light_pos=tuple(p.light_pos))
    hits = 0
    for path in (sr.SR_PATH_FAST, sr.SR_PATH_PLAIN):
        fa = eng.render(idx, u, path=path, aux=True)
        fb = eng.render(UPLOADED, u, path=path, aux=True)
        assert (fa.rgb == fb.rgb).all() and (fa.hit_id == fb.hit_id).all() and (fa.lam == fb.lam).all()
        hits = int((fa.hit_id != 0xFFFFFFFF).sum())
    return hits


def test_device_arena_equals_the_oracle_arena(engine, inputs):
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices)
    A = O.Arena()
    hits = 0
    for k in range(10):
        es = engine_drive(engine, w, k, sc)
        os_ = oracle_drive(A, w, k)
        for key, v in os_.items():
            assert es[key] == v, (k, key, es, os_)
        arrays = assert_same_arena(engine, A)
        assert es["num_nodes"] == len(arrays[0])
        if k in (0, 4, 9):
            hits += assert_same_frames(engine, arrays, p, yaw=90.0 * (k % 4))
    assert hits > 1000


def test_device_arena_rebase_compacts_as_the_oracle(engine, inputs):
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices, n_bodies=12, base=60)
    A = O.Arena()
    idx = IDX + 10
    for k in range(3):
        engine_drive(engine, w, k, sc, idx)
        oracle_drive(A, w, k)
    w.shift = -7.25
    compacted = 0
    for _ in range(3):
        es = engine_drive(engine, w, 3, sc, idx)
        os_ = oracle_drive(A, w, 3)
        assert {k: es[k] for k in os_} == os_
        compacted += es["compacted"]
        arrays = assert_same_arena(engine, A, idx)
    assert compacted == 1
    assert_same_frames(engine, arrays, p, yaw=0.0, idx=idx)


def test_the_reference_flow_patches_the_gpu_copy(engine, inputs):
    """The reference's own dynamic flow on the drop-in boundary: the host arena (the oracle's) is
    patched into the device copy with each edit's dirty ranges through sr_update_scene when the copy
    holds the previous edit of the same layout, else uploaded afresh (update_scene, gpu.rs:704-731);
    the copy then equals the host arena and renders as the device arena does."""
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices)
    A = O.Arena()
    idx = IDX + 20
    version, patched = None, 0
    for k in range(10):
        engine_drive(engine, w, k, sc, idx)
        oracle_drive(A, w, k)
        lay, ed, nr, pr = A.dirty()
        nodes, g, a = A.arrays()
        up = sr.PackedScene(nodes, g, a, p.materials, np.zeros(4, np.float32), 0, tuple(p.light_pos), anchor=p.anchor)
        if version == (lay, ed - 1):
            engine.update(UPLOADED, up, node_ranges=nr, prim_ranges=pr)
            patched += 1
        else:
            engine.upload(UPLOADED, up)
        version = (lay, ed)
        dn, _ = engine.tree(UPLOADED)
        dg, da = engine.records(UPLOADED)
        assert dn.tobytes() == nodes.tobytes() and dg.tobytes() == g.tobytes() and da.tobytes() == a.tobytes()
        if k in (3, 9):
            u = sr.uniforms(sr.camera(fov_deg=100.0, yaw=90.0 * k), 320, 200, 0, 1, 0, num_nodes=len(nodes),
                            light_pos=tuple(p.light_pos))
            for path in (sr.SR_PATH_FAST, sr.SR_PATH_PLAIN):
                fa = engine.render(idx, u, path=path, aux=True)
                fb = engine.render(UPLOADED, u, path=path, aux=True)
                assert (fa.rgb == fb.rgb).all() and (fa.hit_id == fb.hit_id).all()
    assert patched == 9


def test_empty_snapshot_and_restart(engine, inputs):
    """A snapshot with nothing in it leaves the root over nothing (no hits, sky only); a scene
    uploaded or built at the index makes the next snapshot start afresh."""
    sc, tube, simplices, p = inputs
    engine.arena_begin(IDX + 5)
    st = engine.arena_finish(IDX + 5, sc)
    assert st["num_nodes"] == 1 and st["arena_simplices"] == 0
    u = sr.uniforms(sr.camera(), 64, 40, 0, 1, 0, num_nodes=1)
    for path in (sr.SR_PATH_FAST, sr.SR_PATH_PLAIN):
        f = engine.render(IDX + 5, u, path=path, aux=True)
        assert (f.hit_id == 0xFFFFFFFF).all()
    engine.upload(IDX + 5, sc)
    w = W.World(tube, simplices)
    A = O.Arena()
    engine_drive(engine, w, 0, sc, idx=IDX + 5)
    oracle_drive(A, w, 0)
    assert_same_arena(engine, A, idx=IDX + 5)
    with pytest.raises(sr.SrError):
        engine.arena_tube(IDX + 5, (0, 0, 1), sr.TubeData(w.vertices, w.triangles, w.tube_of(0, 0)[0], 0))


def test_a_failed_snapshot_is_undone(engine, inputs):
    """A snapshot that fails before anything is written (here a tube's material id out of range)
    leaves the scene rendering as before, and so does one begun and never finished; the next
    snapshot goes on from the last one written, as the reference's cache would without them."""
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices)
    idx = IDX + 40
    engine_drive(engine, w, 0, sc, idx)
    u = sr.uniforms(sr.camera(fov_deg=100.0), 160, 100, 0, 1, 0, light_pos=tuple(p.light_pos))
    before = engine.render(idx, u, aux=True)
    engine.arena_begin(idx)
    engine.arena_tube(idx, (0, 0, 100), sr.TubeData(w.vertices, w.triangles, w.tube_of(0, 1)[0], 99))
    with pytest.raises(sr.SrError) as e:
        engine.arena_finish(idx, sc)
    assert e.value.status == sr._lib.SR_ERR_BAD_SCENE
    after = engine.render(idx, u, aux=True)
    assert (after.rgb == before.rgb).all() and (after.hit_id == before.hit_id).all()
    engine.arena_begin(idx)
    engine.arena_tube(idx, (0, 0, 101), sr.TubeData(w.vertices, w.triangles, w.tube_of(1, 3)[0], 1))
    A = O.Arena()
    oracle_drive(A, w, 0)
    engine_drive(engine, w, 1, sc, idx)
    oracle_drive(A, w, 1)
    assert_same_arena(engine, A, idx)


def test_a_tube_past_its_rindler_horizon_is_flagged(engine, inputs):
    """Where the reference asserts 1 + a_local . p > 0 (mesh4d.rs:738-751) the tube is extruded all
    the same, as the host builders do, and the snapshot's stats say so."""
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices)
    s, _ = w.tube_of(0, 1)
    s["accel"][3] = (-2.0, 0.0, 0.0)  # 1 + a . p < 0 at the vertices with x = +1.5
    idx = IDX + 45
    A = O.Arena()
    engine.arena_begin(idx)
    engine.arena_tube(idx, (0, 0, 100), sr.TubeData(w.vertices, w.triangles, s, 0))
    st = engine.arena_finish(idx, sc)
    assert st["rindler_crossed"] == 1
    A.begin()
    A.tube((0, 0, 100), w.vertices, w.triangles, s, 0)
    A.finish()
    assert_same_arena(engine, A, idx)
    assert engine.stats(idx).rindler_crossed == 1


def test_tuning_survives_snapshots(engine, inputs):
    """A scene's launch tuning (sr_set_tuning / sr_autotune) stays across snapshots."""
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices)
    idx = IDX + 50
    engine_drive(engine, w, 0, sc, idx)
    t = engine.tuning(idx)
    t.blocks_per_sm = 7
    engine.set_tuning(idx, t)
    engine_drive(engine, w, 1, sc, idx)
    assert engine.tuning(idx).blocks_per_sm == 7


def test_one_chunk_empty_chunks_and_back(engine, inputs):
    """The tree's edge cases as the reference writes them (scene_cache.rs:325-333): nothing (node 0
    over nothing), one chunk (node 0 a copy of its root), an empty piece, many chunks, one again."""
    sc, tube, simplices, p = inputs
    boxes, geoms, attrs = simplices
    idx = IDX + 60
    A = O.Arena()
    steps = [
        [],                                   # nothing
        [(0, [0], slice(0, 25))],             # one chunk
        [(0, [0], slice(0, 25)), (1, [1], slice(30, 30))],   # plus an empty piece
        [(0, [0], slice(0, 25)), (1, [1], slice(30, 30)), (2, [2], slice(40, 75)), (3, [3], slice(80, 81))],
        [(2, [2], slice(40, 75))],            # one again (reused, elsewhere in the arena)
    ]
    for k, pieces in enumerate(steps):
        engine.arena_begin(idx)
        A.begin()
        for i, key, sl in pieces:
            engine.arena_piece(idx, (2, 0, 9), i, key, boxes[sl], geoms[sl], attrs[sl])
            A.piece((2, 0, 9), i, key, boxes[sl], geoms[sl], attrs[sl])
        es = engine.arena_finish(idx, sc)
        os_ = A.finish()
        assert {key: es[key] for key in os_} == os_, k
        arrays = assert_same_arena(engine, A, idx)
        if k in (1, 3, 4):
            assert_same_frames(engine, arrays, p, yaw=0.0, idx=idx)


def test_batches_follow_the_snapshots(engine, inputs):
    """Batched renders replay CUDA graphs keyed by the scene's buffers, which snapshots rewrite and
    regrow: after every snapshot a batch of observers equals their single plain frames."""
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices)
    idx = IDX + 55
    us = []
    for yaw in (0.0, 120.0, 240.0):
        us.append(sr.uniforms(sr.camera(fov_deg=100.0, yaw=yaw), 160, 100, 0, 1, 0, light_pos=tuple(p.light_pos)))
    total = sum(u.size[0] * u.size[1] for u in us)
    hits = 0
    for k in range(6):
        engine_drive(engine, w, k, sc, idx)
        out = np.zeros(total, np.uint32)
        engine.render_batch(idx, us, out.ctypes.data, total, device_output=False)
        off = 0
        for u in us:
            n = u.size[0] * u.size[1]
            ref = engine.render(idx, u, path=sr.SR_PATH_PLAIN, aux=True)
            assert (out[off:off + n] == ref.rgb).all(), k
            hits += int((ref.hit_id != 0xFFFFFFFF).sum())
            off += n
    assert hits > 1000


def test_snapshot_timing(engine, inputs):
    """The per-snapshot cost the reference measures (bench.rs:213-218, rebuild + GPU patch): a world
    of 12 bodies with long histories, three new samples per body per snapshot; the whole
    sr_arena_* sequence timed on the host, against the oracle's host scene cache."""
    sc, tube, simplices, p = inputs
    w = W.World(tube, simplices, n_bodies=12, base=200)
    A = O.Arena()
    idx = IDX + 30
    te, to, stats = [], [], None
    for k in range(8):
        t0 = time.perf_counter()
        stats = engine_drive(engine, w, k, sc, idx)
        te.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        oracle_drive(A, w, k)
        to.append(time.perf_counter() - t0)
    assert_same_arena(engine, A, idx)
    print(f"snapshot of {stats['arena_simplices']} simplices ({stats['simplices_built']} new): device arena "
          f"{np.median(te[2:]) * 1e3:.2f} ms, oracle scene cache on the host {np.median(to[2:]) * 1e3:.2f} ms "
          f"(medians of 6); from an empty cache (every chunk made): device {te[0] * 1e3:.1f} ms, "
          f"host {to[0] * 1e3:.1f} ms")
