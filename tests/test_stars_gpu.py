"""Binned star footprints on the fast path: every frame must equal the brute-force star sum of the
reference's star_light (star.rs:240-286), which the plain path and SR_FLAG_STAR_BRUTE compute,
bit for bit in the HDR image (so also in RGB)."""
import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import packed_from_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def starfield(engine):
    s = O.Scene(O.synth_params(5, 2, n_bodies=8, steps=16, n_stars=20000))
    engine.upload(8, packed_from_oracle(s))
    return s


def _u(scene, cam, w, h, slice_mode=0):
    return sr.uniforms(cam, w, h, 0, 0, slice_mode, num_nodes=int(scene.info.n_nodes),
                       num_stars=int(scene.info.n_stars))


@pytest.mark.parametrize("slice_mode", [0, 1, 2, 3])
def test_binned_equals_brute_single_frame(engine, starfield, slice_mode):
    cam = sr.camera((0.0, 0.0, 0.0, 0.0), 90.0, rapidity=(0.8, -0.3, 0.5))
    u = _u(starfield, cam, 320, 200, slice_mode)
    binned = engine.render(8, u, path=sr.SR_PATH_FAST, hdr=True)
    brute = engine.render(8, u, path=sr.SR_PATH_FAST, hdr=True, star_brute=True)
    plain = engine.render(8, u, path=sr.SR_PATH_PLAIN, hdr=True)
    assert (binned.hdr == brute.hdr).all()
    assert (binned.hdr == plain.hdr).all()
    assert (binned.rgb == plain.rgb).all()
    # The star term is present: the same scene without its stars differs in many pixels.
    p = packed_from_oracle(starfield)
    engine.upload(10, sr.PackedScene(p.nodes, p.geoms, p.attrs, p.materials, p.stars[:4], 0, p.light_pos,
                                     p.leaf_to_orig))
    nostars = engine.render(10, _u(starfield, cam, 320, 200, slice_mode), path=sr.SR_PATH_FAST, hdr=True)
    assert (nostars.hdr != binned.hdr).any(axis=1).sum() > 50


def test_binned_batch_mixed_observers(engine, starfield):
    """A batch mixing binned observers with one whose field of view is too wide for binning (it
    keeps the brute force) and one in another render mode."""
    cams = [(sr.camera((0.0, 0.0, 0.0, 0.0), 90.0, rapidity=(0.8, -0.3, 0.5)), 256, 160, 0),
            (sr.camera((0.0, 1.0, 0.0, -3.0), 60.0, rapidity=(-0.5, 0.9, 0.1), yaw=0.4), 200, 120, 0),
            (sr.camera((0.0, 0.0, 0.0, 0.0), 170.0, rapidity=(0.2, 0.2, 0.2)), 160, 100, 0),
            (sr.camera((0.0, 0.0, 0.0, 0.0), 90.0, rapidity=(1.5, 0.0, 0.0)), 128, 80, 1)]
    us = [sr.uniforms(c, w, h, mode, 0, 0, num_nodes=int(starfield.info.n_nodes),
                      num_stars=int(starfield.info.n_stars)) for c, w, h, mode in cams]
    total = sum(u.size[0] * u.size[1] for u in us)
    out = np.zeros(total, np.uint32)
    engine.render_batch(8, us, out.ctypes.data, total, device_output=False)
    off = 0
    for u in us:
        n = u.size[0] * u.size[1]
        assert (out[off:off + n] == engine.render(8, u, path=sr.SR_PATH_PLAIN).rgb).all()
        off += n


def test_full_starfield_matches_brute(engine):
    """The 100k stars over the cube occluders at 640x400, observer at the target rapidity."""
    s = O.Scene(O.synth_params(5, 1, n_bodies=16, steps=16))
    assert int(s.info.n_stars) == 100000
    engine.upload(9, packed_from_oracle(s))
    cam = sr.camera((0.0, 0.0, 0.0, 0.0), 90.0, rapidity=(0.8, -0.3, 0.5))
    u = sr.uniforms(cam, 640, 400, 0, 0, 0, num_nodes=int(s.info.n_nodes), num_stars=100000)
    binned = engine.render(9, u, path=sr.SR_PATH_FAST, hdr=True, timing=True)
    brute = engine.render(9, u, path=sr.SR_PATH_FAST, hdr=True, timing=True, star_brute=True)
    print("stars ms binned", binned.timings.stars_ms, "shade+stars ms brute", brute.timings.shade_ms)
    assert (binned.hdr == brute.hdr).all()
    assert binned.timings.stars_ms < brute.timings.shade_ms
