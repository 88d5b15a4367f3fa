"""The batched fast path: many observers of one scene in one launch sequence (captured into a CUDA
graph and replayed) must give each observer exactly the frame the single-frame plain path gives,
including after the graph is replayed with new uniforms."""
import ctypes as C

import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import packed_from_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene(engine):
    s = O.Scene(O.synth_params(1, 2))
    engine.upload(3, packed_from_oracle(s))
    return s


def _observers(seed, n, num_nodes, scale=1):
    obs = sr.observers(seed, n)
    us, cams = [], []
    for o in obs:
        w, h = o["width"] // scale, o["height"] // scale
        c = sr.camera(tuple(o["pos"]), 90.0, rapidity=o["rapidity"])
        us.append(sr.uniforms(c, w, h, 0, 1 if o["slice_mode"] == 0 else 2, o["slice_mode"], num_nodes=num_nodes))
        cams.append(sr.cam64(o["pos"], o["rapidity"]))
    return obs, us, cams


def _batch(engine, idx, us, cams=None):
    total = sum(u.size[0] * u.size[1] for u in us)
    out = np.zeros(total, np.uint32)
    engine.render_batch(idx, us, out.ctypes.data, total, cams=cams, device_output=False)
    return out


def test_batch_equals_plain_frames(engine, scene):
    obs, us, _ = _observers(11, 6, int(scene.info.n_nodes), scale=4)
    out = _batch(engine, 3, us)
    off = 0
    for u in us:
        n = u.size[0] * u.size[1]
        ref = engine.render(3, u, path=sr.SR_PATH_PLAIN).rgb
        assert (out[off:off + n] == ref).all()
        off += n


def test_graph_replay_with_new_uniforms(engine, scene):
    for seed in (21, 22, 21):
        obs, us, _ = _observers(seed, 4, int(scene.info.n_nodes), scale=4)
        out = _batch(engine, 3, us)
        off = 0
        for u in us:
            n = u.size[0] * u.size[1]
            assert (out[off:off + n] == engine.render(3, u, path=sr.SR_PATH_PLAIN).rgb).all()
            off += n


def test_fp64_camera_batch_equals_single_frames(engine, scene):
    obs, us, cams = _observers(12, 5, int(scene.info.n_nodes), scale=4)
    out = _batch(engine, 3, us, cams)
    off = 0
    for u, c in zip(us, cams):
        n = u.size[0] * u.size[1]
        ref = engine.render(3, u, path=sr.SR_PATH_PLAIN, cam=c).rgb
        assert (out[off:off + n] == ref).all()
        off += n


@pytest.mark.parametrize("tiling", [(8, 4, 1, 32, 0, 1, 0), (8, 4, 16, 1, 1, 32, 0), (4, 8, 4, 16, 1, 8, 0),
                                    (8, 4, 4, 8, 0, 16, 0), (4, 8, 1, 32, 0, 1, 75), (8, 4, 1, 32, 0, 1, 100)])
def test_every_schedule_gives_the_same_frames(engine, scene, tiling):
    """Chunk size, refill threshold, leaf batching, cooperative leaf tests and per-SM tile bands
    change only the schedule: every
    setting gives the plain path's frames (with shadows, FP64 cameras)."""
    tw, th, chunk, refill, coop, leaf_batch, home = tiling
    keep = engine.tuning(3)
    t = engine.tuning(3)
    t.tile_w, t.tile_h, t.chunk_tiles, t.refill_lanes, t.leaf_coop, t.leaf_batch = tw, th, chunk, refill, coop, leaf_batch
    t.home_pct = home
    t.packet = 0  # the per-ray kernels' schedules
    engine.set_tuning(3, t)
    try:
        obs, us, cams = _observers(13, 4, int(scene.info.n_nodes), scale=4)
        out = _batch(engine, 3, us, cams)
    finally:
        engine.set_tuning(3, keep)
    off = 0
    for u, c in zip(us, cams):
        n = u.size[0] * u.size[1]
        assert (out[off:off + n] == engine.render(3, u, path=sr.SR_PATH_PLAIN, cam=c).rgb).all()
        off += n


@pytest.mark.parametrize("stack,threads,blocks", [(8, 128, 11), (10, 128, 9), (12, 128, 9), (16, 256, 4),
                                                   (12, 512, 3)])
def test_shared_memory_stack_gives_the_same_frames_and_visits(engine, scene, stack, threads, blocks):
    """The lean kernel with the first `stack` traversal-stack entries of each thread in shared
    memory and the rest in local memory (8 entries: many rays go deeper, so both parts are used)
    gives the plain path's frames, and visits exactly the nodes of the oracle's Bvh4D::trace."""
    keep = engine.tuning(3)
    t = engine.tuning(3)
    t.tile_w, t.tile_h, t.chunk_tiles, t.refill_lanes, t.leaf_coop, t.leaf_batch, t.home_pct = 4, 8, 1, 32, 0, 1, 0
    t.block_threads, t.blocks_per_sm, t.stack_smem = threads, blocks, stack
    t.packet = 0
    engine.set_tuning(3, t)
    try:
        obs, us, cams = _observers(14, 4, int(scene.info.n_nodes), scale=4)
        out = _batch(engine, 3, us, cams)
        cam = sr.camera((0.0, 0.0, 0.0, -10.0), 90.0, rapidity=(0.3, 0.1, -0.2))
        u = sr.uniforms(cam, 256, 160, 0, 0, 0, num_nodes=int(scene.info.n_nodes))
        fr = engine.render(3, u, count=True)
    finally:
        engine.set_tuning(3, keep)
    off = 0
    for u_, c in zip(us, cams):
        n = u_.size[0] * u_.size[1]
        assert (out[off:off + n] == engine.render(3, u_, path=sr.SR_PATH_PLAIN, cam=c).rgb).all()
        off += n
    base = O.render(scene, O.make_camera(pos=(0.0, 0.0, 0.0, -10.0), rapidity=(0.3, 0.1, -0.2)),
                    O.make_config(256, 160), stats=True)
    assert fr.timings.nodes_visited == int(base.stats[:, 0].sum())
    assert fr.timings.tets_tested == int(base.stats[:, 2].sum())


def test_invalid_tuning_rejected(engine, scene):
    t = engine.tuning(3)
    t.refill_lanes = 0
    with pytest.raises(sr.SrError):
        engine.set_tuning(3, t)
    t = engine.tuning(3)
    t.stack_smem = 9  # not one of the built depths
    with pytest.raises(sr.SrError):
        engine.set_tuning(3, t)
    t = engine.tuning(3)
    t.packet = 2
    with pytest.raises(sr.SrError):
        engine.set_tuning(3, t)
    t = engine.tuning(3)
    t.packet, t.stack_smem = 1, 12  # the packet form keeps its stack in local memory
    with pytest.raises(sr.SrError):
        engine.set_tuning(3, t)


def test_fast_traversal_visits_the_reference_nodes(engine, scene):
    """The fast path's traversal work equals the oracle's instrumented Bvh4D::trace: the same
    internal nodes and the same tetrahedron tests, frame total."""
    cam = sr.camera((0.0, 0.0, 0.0, -10.0), 90.0, rapidity=(0.3, 0.1, -0.2))
    u = sr.uniforms(cam, 256, 160, 0, 0, 0, num_nodes=int(scene.info.n_nodes))
    fr = engine.render(3, u, count=True)
    base = O.render(scene, O.make_camera(pos=(0.0, 0.0, 0.0, -10.0), rapidity=(0.3, 0.1, -0.2)),
                    O.make_config(256, 160), stats=True)
    assert fr.timings.nodes_visited == int(base.stats[:, 0].sum())
    assert fr.timings.tets_tested == int(base.stats[:, 2].sum())
    assert fr.timings.leaves_visited == int(base.stats[:, 1].sum())


def test_autotune_keeps_frames_identical(engine, scene):
    u = sr.uniforms(sr.camera((0.0, 0.0, 0.0, -5.0), 90.0), 320, 200, 0, 1, 0, num_nodes=int(scene.info.n_nodes))
    before = engine.render(3, u).rgb
    best, ms = engine.autotune(3, u, 1)
    assert ms > 0 and best.tile_w * best.tile_h == 32
    assert (engine.render(3, u).rgb == before).all()


def test_update_scene_patches_ranges(engine):
    """update_scene with dirty ranges gives the same frames as a fresh upload (gpu.rs:704-731)."""
    a = sr.synth_scene(1, 5, n_bodies=8, steps=8).packed()
    b = sr.synth_scene(1, 6, n_bodies=8, steps=8).packed()
    assert len(a.nodes) == len(b.nodes) or True
    engine.upload(4, a)
    u = sr.uniforms(sr.camera((0.0, 0.0, 0.0, -3.0), 90.0), 160, 100, num_nodes=len(b.nodes))
    n_nodes, n_prims = min(len(a.nodes), len(b.nodes)), min(len(a.geoms), len(b.geoms))
    if len(b.nodes) <= len(a.nodes) and len(b.geoms) <= len(a.geoms):
        engine.update(4, b, node_ranges=[(0, len(b.nodes))], prim_ranges=[(0, len(b.geoms))])
    else:
        engine.update(4, b)
    patched = engine.render(4, u).rgb
    engine.upload(4, b)
    fresh = engine.render(4, u).rgb
    assert (patched == fresh).all()
    assert n_nodes > 0 and n_prims > 0


def test_render_update_render_uses_the_new_scene(engine):
    """A frame rendered before sr_update_scene must not leave a captured launch sequence holding the
    old scene's parameters (root box, layout stride, counts): after the update the frames equal a
    fresh upload's."""
    a = sr.synth_scene(1, 5, n_bodies=64, steps=8)
    b = sr.synth_scene(1, 6, n_bodies=48, steps=8)  # fits a's arrays: patched in place
    assert b.num_nodes < a.num_nodes and b.num_prims < a.num_prims
    u = sr.uniforms(sr.camera((0.0, 0.0, 0.0, -3.0), 90.0), 160, 100, num_nodes=b.num_nodes)
    engine.upload(6, a)
    before = engine.render(6, u).rgb
    engine.update(6, b, node_ranges=[(0, b.num_nodes)], prim_ranges=[(0, b.num_prims)])
    after = engine.render(6, u).rgb
    engine.upload(7, b)
    fresh = engine.render(7, u).rgb
    assert (after == fresh).all()
    assert not (before == after).all()


def test_async_output_overlaps_and_equals_the_blocking_batch(engine, scene):
    """SR_FLAG_ASYNC_OUTPUT: batches queued back to back into different pinned framebuffers, each
    readback beside the next batch, equal the blocking batch once synchronized."""
    import torch
    obs, us, cams = _observers(31, 4, int(scene.info.n_nodes), scale=4)
    total = sum(u.size[0] * u.size[1] for u in us)
    ref = _batch(engine, 3, us, cams)
    outs = [torch.zeros(total, dtype=torch.int32, pin_memory=True) for _ in range(3)]
    for o in outs:
        engine.render_batch(3, us, o.data_ptr(), total, cams=cams, device_output=False, async_output=True)
    engine.synchronize()
    for o in outs:
        assert (o.numpy().view(np.uint32) == ref).all()
    with pytest.raises(sr.SrError):
        engine.render_batch(3, us, outs[0].data_ptr(), total, cams=cams, device_output=False, async_output=True,
                            timing=True)


@pytest.mark.parametrize("stack", [0, 12])
def test_compact_layout_gives_the_same_frames_and_visits(engine, scene, stack):
    """The compact node layout (one copy of the child boxes instead of 16 sign-octant copies) gives
    the same frames and visits the same nodes; it takes 15 x 64 bytes less per internal node."""
    from specrel_b200 import _lib as L
    obs, us, cams = _observers(15, 4, int(scene.info.n_nodes), scale=4)
    keep = engine.tuning(3)
    t = engine.tuning(3)
    t.tile_w, t.tile_h, t.chunk_tiles, t.refill_lanes, t.leaf_coop, t.leaf_batch, t.home_pct = 4, 8, 1, 32, 0, 1, 0
    t.stack_smem, t.top_levels, t.packet = stack, 0, 0
    cam = sr.camera((0.0, 0.0, 0.0, -10.0), 90.0, rapidity=(0.3, 0.1, -0.2))
    u = sr.uniforms(cam, 256, 160, 0, 0, 0, num_nodes=int(scene.info.n_nodes))
    engine.set_tuning(3, t)
    try:
        wide = engine.stats(3)
        assert wide.box_copies == 16
        ref = _batch(engine, 3, us, cams)
        ref_work = engine.render(3, u, count=True).timings
        engine.set_layout(3, L.SR_LAYOUT_COMPACT)
        compact = engine.stats(3)
        assert compact.box_copies == 1 and compact.fast_nodes == wide.fast_nodes
        assert wide.device_bytes - compact.device_bytes == 15 * 64 * wide.fast_nodes
        out = _batch(engine, 3, us, cams)
        work = engine.render(3, u, count=True).timings
    finally:
        engine.set_layout(3, L.SR_LAYOUT_AUTO)
        engine.set_tuning(3, keep)
    assert engine.stats(3).box_copies == 16
    assert (out == ref).all()
    assert (work.nodes_visited, work.tets_tested, work.leaves_visited) == \
        (ref_work.nodes_visited, ref_work.tets_tested, ref_work.leaves_visited)


@pytest.mark.parametrize("stack,top", [(0, 4), (0, 8), (12, 6), (12, 8)])
def test_staged_top_levels_give_the_same_frames_and_visits(engine, scene, stack, top):
    """The top `top` levels of the tree read from shared memory (staged per block) instead of
    global memory: the plain path's frames and the oracle's node visits, unchanged."""
    keep = engine.tuning(3)
    t = engine.tuning(3)
    t.tile_w, t.tile_h, t.chunk_tiles, t.refill_lanes, t.leaf_coop, t.leaf_batch, t.home_pct = 4, 8, 1, 32, 0, 1, 0
    t.block_threads, t.blocks_per_sm, t.stack_smem, t.top_levels = 128, 8, stack, top
    t.packet = 0
    engine.set_tuning(3, t)
    try:
        obs, us, cams = _observers(16, 4, int(scene.info.n_nodes), scale=4)
        out = _batch(engine, 3, us, cams)
        cam = sr.camera((0.0, 0.0, 0.0, -10.0), 90.0, rapidity=(0.3, 0.1, -0.2))
        u = sr.uniforms(cam, 256, 160, 0, 0, 0, num_nodes=int(scene.info.n_nodes))
        fr = engine.render(3, u, count=True)
    finally:
        engine.set_tuning(3, keep)
    off = 0  # the batch's frames have shadows on: shadow rays read the staged levels too
    for u_, c in zip(us, cams):
        n = u_.size[0] * u_.size[1]
        assert (out[off:off + n] == engine.render(3, u_, path=sr.SR_PATH_PLAIN, cam=c).rgb).all()
        off += n
    base = O.render(scene, O.make_camera(pos=(0.0, 0.0, 0.0, -10.0), rapidity=(0.3, 0.1, -0.2)),
                    O.make_config(256, 160), stats=True)
    assert fr.timings.nodes_visited == int(base.stats[:, 0].sum())
    assert fr.timings.tets_tested == int(base.stats[:, 2].sum())


def test_invalid_top_levels_rejected(engine, scene):
    for stack, top in ((8, 4), (0, 9), (16, 2)):
        t = engine.tuning(3)
        t.stack_smem, t.top_levels = stack, top
        with pytest.raises(sr.SrError):
            engine.set_tuning(3, t)
