"""The library's caller-side scene pipeline (scene_synth.cpp) against the oracle's restatement of
the reference's (mesh4d.rs, bvh4d.rs, gpu.rs packing): the packed arrays must agree bit for bit,
so every parity test that builds its scene with either gets the same inputs."""
import numpy as np
import pytest

from oracle import oracle as O


def _same(a: np.ndarray, b: np.ndarray, what: str):
    assert a.shape == b.shape, (what, a.shape, b.shape)
    assert a.tobytes() == b.tobytes(), f"{what} differs ({np.count_nonzero(a != b)} items)"


def _compare(config, seed, **kw):
    import specrel_b200 as sr
    prod = sr.synth_scene(config, seed, **kw)
    ok = {k: v for k, v in kw.items() if k in ("n_bodies", "steps", "subdiv", "n_stars")}
    orc = O.Scene(O.synth_params(config, seed, **ok))
    nodes, geoms, attrs, mats, stars, order = orc.pack()
    p = prod.packed()
    _same(p.nodes, nodes, "nodes")
    _same(p.geoms, geoms, "geoms")
    _same(p.attrs, attrs, "attrs")
    _same(p.materials, mats, "materials")
    _same(p.leaf_to_orig, order, "order")
    if orc.info.n_stars:
        _same(p.stars[: len(stars)], stars, "stars")
    assert prod.info.bvh_depth == orc.info.depth
    return prod, orc


def test_config1_cubes_bit_exact():
    prod, orc = _compare(1, 1)
    assert prod.num_prims == 64 * 12 * 64 * 3
    assert prod.info.rindler_ok


def test_config2_icospheres_reduced_bit_exact():
    prod, orc = _compare(2, 7, n_bodies=5, steps=12)
    assert prod.num_prims == 5 * 320 * 12 * 3
    assert list(prod.info.cam_rapidity) == pytest.approx(list(orc.info.cam_rapidity), abs=0)
    assert prod.info.clamped_accel == orc.info.clamped_accel


def test_config5_stars_reduced_bit_exact():
    prod, orc = _compare(5, 2, n_bodies=3, steps=4, n_stars=300)
    assert prod.num_stars == 300


def test_config3_is_config1_on_an_anchor():
    import specrel_b200 as sr
    a = sr.synth_scene(1, 4, n_bodies=3, steps=5).packed()
    b = sr.synth_scene(3, 4, n_bodies=3, steps=5).packed()
    _same(a.geoms, b.geoms, "geoms")
    assert b.anchor == (1e6, 6e4, 0.0, 8e4)


def test_parallel_build_matches_serial():
    import specrel_b200 as sr
    a = sr.synth_scene(2, 11, n_bodies=6, steps=16, threads=1).packed()
    b = sr.synth_scene(2, 11, n_bodies=6, steps=16, threads=8).packed()
    _same(a.nodes, b.nodes, "nodes")
    _same(a.geoms, b.geoms, "geoms")


def test_observers_match():
    import specrel_b200 as sr
    assert sr.observers(5, 64) == O.observers(5, 64)


def test_tables_match_reference_lut():
    import specrel_b200 as sr
    t = sr.tables()
    assert (t[:4096].astype(np.uint8) == O.gamma_lut()).all()
    assert t[4096 + 7 * 13 + 0] == 0b01111  # 'S' first row (hud.rs:491)


@pytest.mark.parametrize("rap", [(0.0, 0.0, 0.0), (0.3, -0.2, 0.5), (1.2, 0.4, -1.1), (-1.9, 0.1, 0.3)])
def test_camera_tetrad_matches_oracle_f32(rap):
    import specrel_b200 as sr
    c = sr.camera((0, 0, 0, 0), 90.0, rapidity=rap)
    mine = np.array([[c.e[a][k] for k in range(4)] for a in range(4)], np.float32)
    ref = O.tetrad(O.make_camera(rapidity=rap), fp64=False).astype(np.float32)
    assert mine.tobytes() == ref.tobytes()


def test_uniforms_build_fields():
    import specrel_b200 as sr
    c = sr.camera((1.0, 2.0, 3.0, 4.0), 65.0)
    u = sr.uniforms(c, 192, 120, mode=3, shadow_mode=1, slice_mode=3, num_nodes=7, num_stars=2,
                    flashes=[((0, 1, 2, 3), 0.8, 2.5, (1.0, 0.9, 0.7))], remote_origins=[(1, 1, 1, 1)])
    assert u.size[0] == 192 and u.size[1] == 120 and u.num_nodes == 7 and u.num_stars == 2
    half_h = np.float32(np.tan(np.float32(0.5) * np.float32(65.0) * (np.float32(np.pi) / np.float32(180))))
    assert abs(u.half_wh[1] - half_h) <= 1e-6
    assert u.num_flashes == 1 and abs(u.flash_col_width[0][0] - 2.5) < 1e-6
    # Prophecy: the camera's own cone first, then the remote frontier (renderer.rs:253-262).
    assert u.num_haze == 2 and tuple(u.haze_origin[0]) == (1.0, 2.0, 3.0, 4.0)
    assert abs(u.frontier_view_offset - 0.14) < 1e-7
