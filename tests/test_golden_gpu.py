"""The engine's plain and fast paths against the committed golden fixtures (tests/golden): hit ids
and (f32 scenes) lambda and tau bit for bit, RGB within 1/255 outside the fixture's near-threshold
mask; for the translated FP64 case, the precision bar of the FP64 rebase (hit ids >= 99.99%,
lambda and tau within 1e-5 relative)."""
import os
import sys

import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import MISS, packed_from_oracle, rgb_diff

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import CASES  # noqa: E402

pytestmark = pytest.mark.gpu

PATHS = [sr.SR_PATH_PLAIN, sr.SR_PATH_FAST]
F32_CASES = sorted(k for k, v in CASES.items() if not v[1])


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("name", F32_CASES)
def test_engine_matches_fixture(engine, name, path):
    sp, _, cam, (w, h, mode, shadow, slice_) = CASES[name]
    g = load(name)
    scene = O.Scene(O.synth_params(**sp))
    engine.upload(6, packed_from_oracle(scene))
    c = sr.camera(cam["pos"], cam.get("fov_deg", 90.0), rapidity=cam.get("rapidity"))
    u = sr.uniforms(c, w, h, mode, shadow, slice_, num_nodes=int(scene.info.n_nodes),
                    num_stars=int(scene.info.n_stars))
    fr = engine.render(6, u, path=path, aux=True)
    assert (fr.hit_id == g["orig"]).all()
    hit = g["orig"] != MISS
    assert (fr.lam[hit] == g["lam"][hit]).all() and (fr.tau[hit] == g["tau"][hit]).all()
    d = rgb_diff(fr.rgb, g["rgb"])
    assert d[~g["near"]].max() <= 1


@pytest.mark.parametrize("path", PATHS)
def test_fp64_rebase_matches_translated_fixture(engine, path):
    name = "config3_translated_fp64_160x100"
    sp, _, cam, (w, h, mode, shadow, slice_) = CASES[name]
    g = load(name)
    scene = sr.synth_scene(3, sp["seed"])
    engine.upload(7, scene)
    u = sr.uniforms(sr.camera(), w, h, mode, shadow, slice_, num_nodes=scene.num_nodes, light_pos=scene.light_pos)
    fr = engine.render(7, u, path=path, aux=True, cam=sr.cam64(cam["pos"]))
    same = fr.hit_id == g["orig"]
    assert same.mean() >= 0.9999
    both = same & (g["orig"] != MISS)
    assert (np.abs(fr.lam[both] - g["lam"][both]) / np.abs(g["lam"][both])).max() <= 1e-5
    assert (np.abs(fr.tau[both] - g["tau"][both]) / np.maximum(np.abs(g["tau"][both]), 1.0)).max() <= 1e-5
    assert (rgb_diff(fr.rgb, g["rgb"]) > 1).mean() <= 0.002
