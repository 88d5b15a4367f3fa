"""The cube scene translated to t = 1e6, |x| = 1e5, observer at the same offset, at 1280x800.

The engine stores the scene's f32 coordinates relative to an FP64 anchor and builds the observer's
event and tetrad in double on the GPU (SrCameraF64), so the f32 traversal runs on small numbers.
It is compared with the all-FP64 oracle render of the translated scene; the naive f32 render of the
translated scene (what the reference's f32 pipeline does) is shown failing for contrast.
"""
import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import MISS, rgb_diff

pytestmark = pytest.mark.gpu

T = (1e6, 6e4, 0.0, 8e4)
W, H = 1280, 800


@pytest.fixture(scope="module")
def fp64_oracle():
    s = O.Scene(O.synth_params(3, 1), fp64=True)
    r = O.render(s, O.make_camera(pos=T), O.make_config(W, H))
    return s, r


def test_fp64_rebase_matches_fp64_oracle(engine, fp64_oracle):
    s64, ref = fp64_oracle
    scene = sr.synth_scene(3, 1)
    assert scene.num_prims == int(s64.info.n_prims)
    engine.upload(5, scene)
    u = sr.uniforms(sr.camera(), W, H, num_nodes=scene.num_nodes, light_pos=scene.light_pos)
    reports = {}
    for path in (sr.SR_PATH_PLAIN, sr.SR_PATH_FAST):
        fr = engine.render(5, u, path=path, aux=True, cam=sr.cam64(T))
        same = fr.hit_id == ref.orig
        hit = (ref.orig != MISS) & same
        lam_rel = np.abs(fr.lam[hit] - ref.lam[hit]) / np.abs(ref.lam[hit])
        tau_rel = np.abs(fr.tau[hit] - ref.tau[hit]) / np.maximum(np.abs(ref.tau[hit]), 1.0)
        d = rgb_diff(fr.rgb, ref.rgb)
        reports[path] = dict(hit_agree=float(same.mean()), lam_max=float(lam_rel.max()),
                             lam_med=float(np.median(lam_rel)), tau_max=float(tau_rel.max()),
                             tau_med=float(np.median(tau_rel)), rgb_max=int(d.max()),
                             rgb_gt1=float((d > 1).mean()))
        print(path, reports[path])
        assert same.mean() >= 0.9999
        assert lam_rel.max() <= 1e-5 and tau_rel.max() <= 1e-5
        assert d.max() <= 1  # every pixel within 1/255 of the FP64 oracle (measured: max 1)
    # The two engine paths agree with each other exactly.
    assert reports[0] == reports[1]


def test_naive_f32_translated_scene_fails(fp64_oracle):
    """Without the rebase (f32 coordinates at t = 1e6) the hits are wrong: the reason for the
    FP64 anchor."""
    s64, ref = fp64_oracle
    s32 = O.Scene(O.synth_params(3, 1))
    r32 = O.render(s32, O.make_camera(pos=T), O.make_config(W, H))
    agree = float((r32.orig == ref.orig).mean())
    print("naive f32 hit agreement", agree)
    assert agree < 0.999
