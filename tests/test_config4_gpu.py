"""The batched-observer workload at its stated size: the cube scene (64 inertial cubes, 147k tets)
seen by the seeded batch of 64 observers (resolutions 320x200 .. 1920x1200, past light cone and
God's-eye slice, rapidities |phi| <= 3), rendered in ONE sr_render_batch call, as bench.py times it.

Five observers of the batch are held to the oracle at full resolution (a 1920x1200 past-cone and a
1920x1200 God's-eye frame, a 1280x800 past-cone, a 640x400 God's-eye and a 320x200 past-cone; of
each kind the one that sees the most geometry: the workload's unit cubes are spread over a 40-unit
box, so most of every frame is sky), in both camera forms:
- the reference's f32 camera (uniforms only): the batch's RGB against the f32 oracle, at the
  parity bar (RGB8 within 1/255 outside the near-threshold mask; fewer than 0.5% of pixels more
  than 4 off), and the same observer's hit ids, lambda and tau from the fast path against the
  oracle's (ids equal on non-grazing rays, lambda and tau within 1e-5 relative);
- the FP64 camera (SrCameraF64, what the bench measures): against the all-FP64 oracle (scene built
  and rendered in double): hit-id agreement >= 99.99%, and no further from it than the reference's
  own f32 renderer (the f32 oracle) is: lambda and tau errors on agreeing hits within the f32
  renderer's (or 1e-5, if that is larger), and no more pixels more than 1/255 off. With observers
  up to 50 light-seconds from the origin at rapidities up to 3, f32 arithmetic moves texture edges
  (clock hands, digits, grid lines) against FP64: the f32 renderer itself shows up to 166 such
  pixels and lambda errors up to 5e-4 on these frames.
"""
import os

import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import MISS, compare, oracle_frames, packed_from_oracle, rgb_diff

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
PICK = [50, 1, 13, 63, 57]  # 1920x1200 cone, 1920x1200 God's-eye, 1280x800 cone, 640x400 God's-eye, 320x200 cone
# Near-threshold mask fractions of these frames as measured (the oracle is deterministic) and the
# share of pixels that hit a tetrahedron.
NEAR = {50: 1.085e-05, 1: 2.387e-05, 13: 2.637e-05, 63: 7.81e-06, 57: 1.563e-05}
HITS = {50: 0.0055, 1: 0.0122, 13: 0.0079, 63: 0.057, 57: 0.0298}


def _shadow(slice_mode):
    return 1 if slice_mode == 0 else 2


@pytest.fixture(scope="module")
def batch(engine):
    s32 = O.Scene(O.synth_params(1, 1))
    s64 = O.Scene(O.synth_params(1, 1), fp64=True)
    engine.upload(30, packed_from_oracle(s32))
    obs = O.observers(1, 64)
    assert obs == sr.observers(1, 64)
    nn = int(s32.info.n_nodes)
    us = [sr.uniforms(sr.camera(o["pos"], 90.0, rapidity=o["rapidity"]), o["width"], o["height"], 0,
                      _shadow(o["slice_mode"]), o["slice_mode"], num_nodes=nn) for o in obs]
    cams = [sr.cam64(o["pos"], o["rapidity"]) for o in obs]
    total = sum(u.size[0] * u.size[1] for u in us)
    offs = np.cumsum([0] + [u.size[0] * u.size[1] for u in us])
    f32 = np.zeros(total, np.uint32)
    f64 = np.zeros(total, np.uint32)
    engine.render_batch(30, us, f32.ctypes.data, total, device_output=False)
    engine.render_batch(30, us, f64.ctypes.data, total, cams=cams, device_output=False)
    return dict(s32=s32, s64=s64, obs=obs, us=us, cams=cams, offs=offs, f32=f32, f64=f64)


@pytest.mark.parametrize("i", PICK)
def test_batch_observer_against_f32_oracle(engine, batch, i):
    o, u = batch["obs"][i], batch["us"][i]
    cfg = O.make_config(o["width"], o["height"], 0, _shadow(o["slice_mode"]), o["slice_mode"])
    base, near = oracle_frames(batch["s32"], O.make_camera(pos=o["pos"], rapidity=o["rapidity"]), cfg, threads=THREADS)
    fr = engine.render(30, u, path=sr.SR_PATH_FAST, aux=True)
    fr.rgb = batch["f32"][batch["offs"][i]:batch["offs"][i + 1]]  # the batch's own pixels
    rep = compare(fr, base, near)
    print(f"observer {i} {o['width']}x{o['height']} slice {o['slice_mode']}, f32 camera, batch:", rep)
    assert rep.hit_match_nongrazing == 1.0 and rep.hit_match >= 0.9999
    assert rep.lam_max_rel <= 1e-5 and rep.tau_max_rel <= 1e-5
    assert rep.rgb_max_unmasked <= 1
    assert rep.frac_gt4 < 0.005
    assert abs(rep.near_threshold_frac - NEAR[i]) <= 0.1 * NEAR[i] + 1e-6, rep.near_threshold_frac
    assert abs((fr.hit_id != MISS).mean() - HITS[i]) <= 0.1 * HITS[i]


@pytest.mark.parametrize("i", PICK)
def test_batch_observer_fp64_camera_against_fp64_oracle(engine, batch, i):
    o, u = batch["obs"][i], batch["us"][i]
    cfg = O.make_config(o["width"], o["height"], 0, _shadow(o["slice_mode"]), o["slice_mode"])
    cam = O.make_camera(pos=o["pos"], rapidity=o["rapidity"])
    ref = O.render(batch["s64"], cam, cfg, threads=THREADS)
    f32, near = oracle_frames(batch["s32"], cam, cfg, threads=THREADS)  # the reference's f32 renderer
    fr = engine.render(30, u, path=sr.SR_PATH_FAST, aux=True, cam=batch["cams"][i])
    rgb = batch["f64"][batch["offs"][i]:batch["offs"][i + 1]]

    def errors(ids, lam, tau, colours):
        ids = ids.astype(np.uint32)
        same = ids == ref.orig.astype(np.uint32)
        hit = same & (ids != MISS)
        lr = np.abs(lam[hit].astype(np.float64) - ref.lam[hit]) / np.abs(ref.lam[hit])
        tr = np.abs(tau[hit].astype(np.float64) - ref.tau[hit]) / np.maximum(np.abs(ref.tau[hit]), 1.0)
        d = rgb_diff(colours, ref.rgb)
        return (same, lr.max() if lr.size else 0.0, tr.max() if tr.size else 0.0, int((d[same & ~near] > 1).sum()),
                int(d.max()))

    same, lam, tau, flips, dmax = errors(fr.hit_id, fr.lam, fr.tau, rgb)
    same32, lam32, tau32, flips32, dmax32 = errors(f32.orig, f32.lam, f32.tau, f32.rgb)
    print(f"observer {i} {o['width']}x{o['height']} slice {o['slice_mode']} vs FP64 oracle: FP64-camera batch: hits "
          f"{same.mean() * 100:.5f}%, lambda rel max {lam:.2e}, tau rel max {tau:.2e}, pixels > 1/255 off {flips} "
          f"(max {dmax}); the f32 renderer: hits {same32.mean() * 100:.5f}%, lambda {lam32:.2e}, tau {tau32:.2e}, "
          f"pixels > 1/255 off {flips32} (max {dmax32})")
    assert same.mean() >= 0.9999
    assert lam <= max(lam32, 1e-5) and tau <= max(tau32, 1e-5)
    assert flips <= flips32
    # The batch's pixels are the single-frame fast path's.
    assert (rgb == fr.rgb).all()
