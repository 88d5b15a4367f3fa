"""At full size: the 7.9M-tet accelerated-icosphere scene at 1280x800, the workload's own
observer (the bench's first frame), on the fast (batched) path.

- With the reference's f32 camera, against the f32 oracle on the same packed scene: hit ids,
  lambda and tau bit-identical, RGB8 within 1/255 outside the near-threshold mask (the parity bar,
  at full size).
- With the FP64 camera (the batched FP32 + FP64-rebase configuration the bench measures), against
  the all-FP64 oracle (scene built and rendered in double): the hit-id agreement bar
  (>= 99.99%) and colour within 1/255 on agreeing pixels outside the near-threshold mask, with the
  lambda and tau errors reported. The f32-camera frame is measured against the FP64 oracle too.
The printed lines are the measurement quoted for this configuration.
"""
import os

import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import MISS, compare, oracle_frames, packed_from_oracle, rgb_diff

pytestmark = pytest.mark.gpu

W, H = 1280, 800
THREADS = os.cpu_count() or 1
# (rapidity, yaw in degrees, slice mode): 0 past light cone, 1 God's-eye, 2 future light cone.
VIEWS = [((2.8, 0.0, 0.0), 0.0, 0), ((-2.9, 0.4, 0.5), 35.0, 0), ((0.0, -2.5, 1.0), 0.0, 1),
         ((1.5, 1.5, 1.5), -20.0, 2)]


@pytest.fixture(scope="module")
def full(engine):
    s32 = O.Scene(O.synth_params(2, 1))
    engine.upload(20, packed_from_oracle(s32))
    rap = tuple(s32.info.cam_rapidity)
    cfg = O.make_config(W, H, 0, 1, 0)
    base, near = oracle_frames(s32, O.make_camera(rapidity=rap), cfg, threads=THREADS)
    u = sr.uniforms(sr.camera(rapidity=rap), W, H, 0, 1, 0, num_nodes=int(s32.info.n_nodes))
    # The three bench observers with the largest rapidities (the fastest ray axes), rendered by the
    # f32 oracle too.
    from specrel_b200 import shard
    raps = shard.observer_rapidities(1, 0, 8, rap)[1:]
    fast = sorted(raps, key=lambda r: -float(np.dot(r, r)))[:3]
    boosted = [(r,) + oracle_frames(s32, O.make_camera(rapidity=r), cfg, threads=THREADS) for r in fast]
    # Views beyond the bench's: rapidities up to |phi| = 3, the God's-eye and future-cone slices, a
    # turned camera.
    views = []
    for r, yaw, slice_mode in VIEWS:
        c = O.make_config(W, H, 0, 1 if slice_mode == 0 else 2, slice_mode)
        views.append((r, yaw, slice_mode) + oracle_frames(s32, O.make_camera(rapidity=r, yaw=yaw), c, threads=THREADS))
    del s32
    f32 = engine.render(20, u, path=sr.SR_PATH_FAST, aux=True)
    f64 = engine.render(20, u, path=sr.SR_PATH_FAST, aux=True, cam=sr.cam64((0.0, 0.0, 0.0, 0.0), rap))
    return dict(rap=rap, cfg=cfg, base=base, near=near, f32=f32, f64=f64, u=u, n_nodes=int(u.num_nodes),
                boosted=boosted, views=views)


@pytest.fixture(scope="module")
def fp64_ref(full):
    s64 = O.Scene(O.synth_params(2, 1), fp64=True)
    ref = O.render(s64, O.make_camera(rapidity=full["rap"]), full["cfg"], threads=THREADS)
    del s64
    return ref


def test_full_frame_equals_f32_oracle(full):
    rep = compare(full["f32"], full["base"], full["near"])
    print("7.9M tets 1280x800, f32 camera vs f32 oracle:", rep)
    assert rep.hit_match == 1.0
    assert rep.lam_max_rel == 0.0 and rep.tau_max_rel == 0.0
    assert rep.rgb_max_unmasked <= 1
    assert full["f32"].timings.shadow_rays > 10000


def _against_fp64(fr, ref, near, label):
    gid = fr.hit_id.astype(np.uint32)
    same = gid == ref.orig.astype(np.uint32)
    hit = same & (gid != MISS)
    lam_rel = np.abs(fr.lam[hit].astype(np.float64) - ref.lam[hit]) / np.abs(ref.lam[hit])
    tau_rel = np.abs(fr.tau[hit].astype(np.float64) - ref.tau[hit]) / np.maximum(np.abs(ref.tau[hit]), 1.0)
    d = rgb_diff(fr.rgb, ref.rgb)
    ok = same & ~near
    print(f"7.9M tets 1280x800, {label} vs FP64 oracle: hit-id agreement {same.mean() * 100:.5f}% "
          f"({int((~same).sum())} of {same.size} differ), lambda rel max {lam_rel.max():.2e} median "
          f"{np.median(lam_rel):.2e}, tau rel max {tau_rel.max():.2e} median {np.median(tau_rel):.2e}, "
          f"rgb max {int(d.max())}, on agreeing pixels outside the near-threshold mask {int(d[ok].max())} "
          f"(> 1 on {int((d[ok] > 1).sum())}), near-threshold {near.mean() * 100:.3f}%")
    return same, lam_rel, tau_rel, d, ok


def test_fp64_camera_frame_against_fp64_oracle(full, fp64_ref):
    same, lam_rel, tau_rel, d, ok = _against_fp64(full["f64"], fp64_ref, full["near"], "FP64 camera")
    assert same.mean() >= 0.9999
    assert lam_rel.max() <= 1e-5 and tau_rel.max() <= 1e-5
    assert d[ok].max() <= 1


def test_f32_camera_frame_against_fp64_oracle(full, fp64_ref):
    same, lam_rel, tau_rel, d, ok = _against_fp64(full["f32"], fp64_ref, full["near"], "f32 camera")
    assert same.mean() >= 0.9999
    assert d[ok].max() <= 1


def test_packet_traversal_at_full_size(engine, full):
    """The packet traversal (SrTuning.packet = 1) on the full-size scene: the workload's own frame
    bit-identical to the f32 oracle, and the bench's other seven observers (FP64 cameras) identical
    to the per-ray order in hit record, lambda and tau."""
    from specrel_b200 import shard
    keep = engine.tuning(20)

    def with_packet(on, fn):
        t = engine.tuning(20)
        t.packet = on
        engine.set_tuning(20, t)
        return fn()

    try:
        fr = with_packet(1, lambda: engine.render(20, full["u"], path=sr.SR_PATH_FAST, aux=True))
        rep = compare(fr, full["base"], full["near"])
        print("7.9M tets 1280x800, packet traversal, f32 camera vs f32 oracle:", rep)
        assert rep.hit_match == 1.0 and rep.lam_max_rel == 0.0 and rep.tau_max_rel == 0.0
        assert rep.rgb_max_unmasked <= 1
        for r in shard.observer_rapidities(1, 0, 8, full["rap"])[1:]:
            u = sr.uniforms(sr.camera(rapidity=r), W, H, 0, 1, 0, num_nodes=full["n_nodes"])
            c = sr.cam64((0.0, 0.0, 0.0, 0.0), r)
            a = with_packet(1, lambda: engine.render(20, u, path=sr.SR_PATH_FAST, aux=True, cam=c))
            b = with_packet(0, lambda: engine.render(20, u, path=sr.SR_PATH_FAST, aux=True, cam=c))
            assert (a.hit_id == b.hit_id).all()
            assert (a.lam.view(np.uint32) == b.lam.view(np.uint32)).all()
            assert (a.tau.view(np.uint32) == b.tau.view(np.uint32)).all()
            assert (a.rgb == b.rgb).all()
    finally:
        engine.set_tuning(20, keep)


def test_boosted_observers_equal_f32_oracle(engine, full):
    """The bench's three most boosted observers (|phi| up to 2: the rays' fastest axes, where the
    packet walk's margin between a hit and its leaf box's entry is thinnest) on the default fast
    path (the packet traversal) against the f32 oracle at full size: hit ids, lambda and tau bit for
    bit, RGB8 within 1/255 outside the near-threshold mask."""
    assert engine.tuning(20).packet == 1
    for r, base, near in full["boosted"]:
        u = sr.uniforms(sr.camera(rapidity=r), W, H, 0, 1, 0, num_nodes=full["n_nodes"])
        rep = compare(engine.render(20, u, path=sr.SR_PATH_FAST, aux=True), base, near)
        print(f"7.9M tets 1280x800, rapidity |phi| = {float(np.linalg.norm(r)):.2f}, packet vs f32 oracle:", rep)
        assert rep.hit_match == 1.0 and rep.lam_max_rel == 0.0 and rep.tau_max_rel == 0.0
        assert rep.rgb_max_unmasked <= 1


def test_sweep_of_views_equals_f32_oracle(engine, full):
    """Views beyond the bench's observers on the default fast path (the packet traversal) against
    the f32 oracle at full size: rapidities up to |phi| = 3, the God's-eye and future-cone slices, a
    turned camera. Hit ids, lambda and tau bit for bit, RGB8 within 1/255 outside the mask."""
    for r, yaw, slice_mode, base, near in full["views"]:
        u = sr.uniforms(sr.camera(rapidity=r, yaw=yaw), W, H, 0, 1 if slice_mode == 0 else 2, slice_mode,
                        num_nodes=full["n_nodes"])
        rep = compare(engine.render(20, u, path=sr.SR_PATH_FAST, aux=True), base, near)
        print(f"7.9M tets 1280x800, rapidity {r}, yaw {yaw}, slice {slice_mode}, packet vs f32 oracle:", rep)
        assert rep.hit_match == 1.0 and rep.lam_max_rel == 0.0 and rep.tau_max_rel == 0.0
        assert rep.rgb_max_unmasked <= 1
