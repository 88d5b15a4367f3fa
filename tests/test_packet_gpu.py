"""The packet traversal (SrTuning.packet = 1): each warp walks its tile's 32 primary rays as one
packet, one node sequence for all of them, each lane with its own closest hit. Every ray must get the
hit the per-ray near-first order gives (the reference's Bvh4D::trace, bvh4d.rs:445-520): the same
record, lambda and tau bit for bit, and so the same frames, in both node layouts; hits at equal
lambda in different leaves must resolve as the reference's order meets them."""
import ctypes as C

import numpy as np
import pytest

import specrel_b200 as sr
from specrel_b200 import _lib as L
from oracle import oracle as O
from parity import packed_from_oracle

pytestmark = pytest.mark.gpu

IDX, TIES = 5, 6


@pytest.fixture(scope="module")
def scene(engine):
    s = O.Scene(O.synth_params(1, 2))
    engine.upload(IDX, packed_from_oracle(s))
    return s


def _tuning(engine, idx, **kw):
    t = engine.tuning(idx)
    for k, v in kw.items():
        setattr(t, k, v)
    engine.set_tuning(idx, t)


def _observers(seed, n, num_nodes, scale):
    us, cams = [], []
    for o in sr.observers(seed, n):
        c = sr.camera(tuple(o["pos"]), 90.0, rapidity=o["rapidity"])
        us.append(sr.uniforms(c, o["width"] // scale, o["height"] // scale, 0, 1 if o["slice_mode"] == 0 else 2,
                              o["slice_mode"], num_nodes=num_nodes))
        cams.append(sr.cam64(o["pos"], o["rapidity"]))
    return us, cams


def _batch(engine, idx, us, cams):
    total = sum(u.size[0] * u.size[1] for u in us)
    out = np.zeros(total, np.uint32)
    engine.render_batch(idx, us, out.ctypes.data, total, cams=cams, device_output=False)
    return out


def _aux_equal(a, b):
    assert (a.hit_id == b.hit_id).all()
    assert (a.lam.view(np.uint32) == b.lam.view(np.uint32)).all()
    assert (a.tau.view(np.uint32) == b.tau.view(np.uint32)).all()
    assert (a.rgb == b.rgb).all()


@pytest.mark.parametrize("layout", [L.SR_LAYOUT_OCTANT, L.SR_LAYOUT_COMPACT])
@pytest.mark.parametrize("tile", [(4, 8), (8, 4)])
def test_packet_frames_equal_per_ray_frames(engine, scene, layout, tile):
    """Mixed observers (past cone, God's-eye, future cone, prophecy; FP64 cameras; shadows): the
    packet batch equals the per-ray batch and the plain path, and single frames carry the same hit
    records, lambda and tau."""
    keep = engine.tuning(IDX)
    engine.set_layout(IDX, layout)
    try:
        us, cams = _observers(31, 6, int(scene.info.n_nodes), 2)
        _tuning(engine, IDX, tile_w=tile[0], tile_h=tile[1], packet=0)
        per_ray = _batch(engine, IDX, us, cams)
        _tuning(engine, IDX, packet=1)
        packet = _batch(engine, IDX, us, cams)
        assert (packet == per_ray).all()
        off = 0
        for u, c in zip(us, cams):
            n = u.size[0] * u.size[1]
            assert (packet[off:off + n] == engine.render(IDX, u, path=sr.SR_PATH_PLAIN, cam=c).rgb).all()
            off += n
        for u, c in zip(us[:3], cams[:3]):
            _aux_equal(engine.render(IDX, u, path=sr.SR_PATH_FAST, aux=True, cam=c),
                       engine.render(IDX, u, path=sr.SR_PATH_PLAIN, aux=True, cam=c))
    finally:
        engine.set_tuning(IDX, keep)
        engine.set_layout(IDX, L.SR_LAYOUT_AUTO)


def test_packet_tuning_needs_the_plain_schedule(engine, scene):
    t = engine.tuning(IDX)
    t.packet, t.top_levels = 1, 4
    with pytest.raises(sr.SrError):
        engine.set_tuning(IDX, t)
    t = engine.tuning(IDX)
    t.packet, t.refill_lanes = 1, 16
    with pytest.raises(sr.SrError):
        engine.set_tuning(IDX, t)


def tie_scene():
    """The cube scene with every simplex twice: the copy has the same hot and cold records (so every
    hit is a hit of both at the same lambda) but a box stretched to one side (still holding the
    simplex), so the copies sit elsewhere in the tree and equal-lambda hits meet in different
    leaves. Built on the host (sr_bvh_build_host) and packed in leaf order."""
    boxes, geoms, attrs, p = sr.synth_scene(1, 2).build_inputs()
    n = len(boxes)
    ext = boxes[:, 4:] - boxes[:, :4]
    dup = boxes.copy()
    dup[:, 1] -= 1.5 * ext[:, 1]  # x min pushed out
    dup[:, 7] += 0.7 * ext[:, 3]  # z max pushed out
    b2 = np.ascontiguousarray(np.concatenate([boxes, dup]), np.float32)
    g2, a2 = np.concatenate([geoms, geoms]), np.concatenate([attrs, attrs])
    nodes = np.zeros(2 * (2 * n) - 1, L.NODE_DTYPE)
    order = np.zeros(2 * n, np.uint32)
    nn, med = C.c_uint32(), C.c_uint32()
    assert L.lib().sr_bvh_build_host(b2.ctypes.data, 2 * n, 8, nodes.ctypes.data, len(nodes), order.ctypes.data,
                                     C.byref(nn), C.byref(med)) == L.SR_OK
    packed = sr.PackedScene(nodes[:nn.value].copy(), g2[order], a2[order], p.materials, p.stars, 0, p.light_pos,
                            order.copy())
    return packed, n


def test_equal_lambda_hits_resolve_in_the_reference_order(engine):
    packed, n = tie_scene()
    engine.upload(TIES, packed)
    keep = engine.tuning(TIES)
    try:
        us, cams = _observers(32, 4, len(packed.nodes), 2)
        seen_copy = seen_orig = 0
        for packet in (0, 1):
            _tuning(engine, TIES, packet=packet)
            for u, c in zip(us, cams):
                fast = engine.render(TIES, u, path=sr.SR_PATH_FAST, aux=True, cam=c)
                _aux_equal(fast, engine.render(TIES, u, path=sr.SR_PATH_PLAIN, aux=True, cam=c))
                hit = fast.hit_id != 0xFFFFFFFF
                seen_copy += int((fast.hit_id[hit] >= n).sum())
                seen_orig += int((fast.hit_id[hit] < n).sum())
        # Both members of the pairs win somewhere: the order between leaves decides, not the index.
        assert seen_copy > 100 and seen_orig > 100
    finally:
        engine.set_tuning(TIES, keep)


@pytest.mark.parametrize("threads,blocks", [(64, 16), (256, 4), (512, 2)])
def test_packet_block_shapes_give_the_same_frames(engine, scene, threads, blocks):
    """The packet kernels (primary rays and the main light's shadow rays) in other block shapes:
    the per-ray frames and the plain path's hit records."""
    keep = engine.tuning(IDX)
    try:
        us, cams = _observers(33, 4, int(scene.info.n_nodes), 2)
        _tuning(engine, IDX, packet=0)
        per_ray = _batch(engine, IDX, us, cams)
        _tuning(engine, IDX, packet=1, block_threads=threads, blocks_per_sm=blocks)
        assert (_batch(engine, IDX, us, cams) == per_ray).all()
        u, c = us[0], cams[0]
        _aux_equal(engine.render(IDX, u, path=sr.SR_PATH_FAST, aux=True, cam=c),
                   engine.render(IDX, u, path=sr.SR_PATH_PLAIN, aux=True, cam=c))
    finally:
        engine.set_tuning(IDX, keep)


def test_packet_on_a_one_leaf_tree_and_tiny_frames(engine, scene):
    """Edge cases of the packet walk against the per-ray and plain paths, hit records bit for bit:
    a tree that is a single leaf (three records the cube scene's camera hits, so every ray tests
    all of them in one leaf), and frames smaller than a tile or not a multiple of it (1x1, 3x5,
    7x9, 33x17), where a warp's lanes outside the frame take no part."""
    cam = sr.camera((0.0, 0.0, 0.0, 0.0), 90.0)
    u = sr.uniforms(cam, 160, 100, 0, 1, 0, num_nodes=int(scene.info.n_nodes))
    full = engine.render(IDX, u, path=sr.SR_PATH_PLAIN, aux=True)
    ids = np.unique(full.hit_id[full.hit_id != 0xFFFFFFFF])
    assert len(ids) >= 3
    boxes, geoms, attrs, p = sr.synth_scene(1, 2).build_inputs()
    pick = ids[np.linspace(0, len(ids) - 1, 3).astype(int)]
    b = np.ascontiguousarray(boxes[pick], np.float32)
    nodes = np.zeros(5, L.NODE_DTYPE)
    order = np.zeros(3, np.uint32)
    nn, med = C.c_uint32(), C.c_uint32()
    assert L.lib().sr_bvh_build_host(b.ctypes.data, 3, 1, nodes.ctypes.data, len(nodes), order.ctypes.data,
                                     C.byref(nn), C.byref(med)) == L.SR_OK
    assert nn.value == 1 and nodes[0]["count"] == 3  # the root is the one leaf
    tiny = sr.PackedScene(nodes[:1].copy(), geoms[pick][order], attrs[pick][order], p.materials, p.stars, 0,
                          p.light_pos, order.copy())
    engine.upload(TIES, tiny)
    keep = engine.tuning(TIES)
    try:
        for packet in (0, 1):
            _tuning(engine, TIES, packet=packet)
            f = engine.render(TIES, sr.uniforms(cam, 160, 100, 0, 1, 0, num_nodes=1), path=sr.SR_PATH_FAST, aux=True)
            _aux_equal(f, engine.render(TIES, sr.uniforms(cam, 160, 100, 0, 1, 0, num_nodes=1), path=sr.SR_PATH_PLAIN,
                                        aux=True))
            assert (f.hit_id != 0xFFFFFFFF).sum() > 0
    finally:
        engine.set_tuning(TIES, keep)
    keep = engine.tuning(IDX)
    try:
        for w, h in ((1, 1), (3, 5), (7, 9), (33, 17)):
            uw = sr.uniforms(sr.camera((0.0, 0.0, 0.0, -10.0), 40.0, rapidity=(0.2, 0.0, 0.1)), w, h, 0, 1, 0,
                             num_nodes=int(scene.info.n_nodes))
            ref = engine.render(IDX, uw, path=sr.SR_PATH_PLAIN, aux=True)
            for packet in (0, 1):
                _tuning(engine, IDX, packet=packet)
                _aux_equal(engine.render(IDX, uw, path=sr.SR_PATH_FAST, aux=True), ref)
    finally:
        engine.set_tuning(IDX, keep)
