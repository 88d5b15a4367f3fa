"""The reference's end-to-end known answers through the engine: the demo scenes the oracle restates
from src/scene.rs, uploaded through the C ABI, must pass the reference's physics probes with the
reference's bars (scene.rs:785-1053) via sr_trace_rays, every probe ray giving the oracle's hit,
lambda and proper time bit for bit; and rendered through sr_render_ex, they must show no black
pixel (scene.rs:733-754), the flash after a round trip (scene.rs:757-782), and the oracle's frames
at the parity bar."""
import numpy as np
import pytest

import probes as P
import specrel_b200 as sr
from oracle import oracle as O
from parity import compare, oracle_frames

pytestmark = pytest.mark.gpu

BASE = 40  # scene slots of this module: BASE + demo id


def _light4(s):
    return (0.0, *s.light)


@pytest.fixture(scope="module")
def demos(engine):
    out = {}
    for w in range(6):
        s = O.Scene.demo(w)
        nodes, geoms, attrs, mats, stars, order = s.pack()
        engine.upload(BASE + w, sr.PackedScene(nodes, geoms, attrs, mats, stars, int(s.info.n_stars), _light4(s), order))
        out[w] = s
    return out


def _tracer(engine, demos, w, log):
    return P.checked_tracer(P.engine_tracer(engine, BASE + w), P.oracle_tracer(demos[w]), log)


def test_twin_paradox_differential_clock_aging(engine, demos):
    log = []
    home, trav = P.twin_aging(_tracer(engine, demos, O.DEMO_TWIN_PARADOX, log))
    print("engine: home", home, "traveler", trav)
    assert log


def test_barn_and_pole_world_slice_vs_camera_slice(engine, demos):
    print("engine:", P.barn_and_pole(_tracer(engine, demos, O.DEMO_BARN_AND_POLE, [])))


def test_einstein_train_all_wagons_visible_and_synced(engine, demos):
    print("engine: max tau error", P.train_sync(_tracer(engine, demos, O.DEMO_EINSTEIN_TRAIN, [])))


def test_loop_boundary_past_light_cone_continuity(engine, demos):
    s = demos[O.DEMO_BARN_AND_POLE]
    print("engine:", P.loop_continuity(_tracer(engine, demos, O.DEMO_BARN_AND_POLE, []), s.window))


def test_penrose_sphere_circular_silhouette(engine, demos):
    log = []
    radii, dev = P.penrose_circularity(_tracer(engine, demos, O.PENROSE_SPHERE, log))
    print("engine: radii", radii, "max deviation", dev, "rays", sum(log))


def test_ray_query_edge_cases(engine, demos):
    """Misses, an empty interval and no rays at all."""
    h = engine.trace_rays(BASE + O.DEMO_TWIN_PARADOX, np.stack([P.ray((15.0, -1.2, -1.05, 0.0), P.Z, 0.1, 0.5),
                                                               P.ray((15.0, -1.2, -1.05, 0.0), P.Z, 2.0, 1.0),
                                                               P.ray((15.0, 90.0, 90.0, 0.0), P.Z, 0.1, 20.0)]))
    assert (h["id"] == P.MISS).all() and (h["slot"] == P.MISS).all()
    assert len(engine.trace_rays(BASE + O.DEMO_TWIN_PARADOX, np.zeros((0, 10)))) == 0
    with pytest.raises(sr.SrError):
        engine.trace_rays(99, np.zeros((1, 10)))


@pytest.mark.parametrize("path", [sr.SR_PATH_PLAIN, sr.SR_PATH_FAST])
def test_all_five_paradox_scenes_render(engine, demos, path):
    """Every static demo scene at 80x50 (shaded, Lorentz-invariant shadows, past light cone): no black
    pixel, and the oracle's frame at the parity bar."""
    for w in range(5):
        s = demos[w]
        cam = s.initial_camera
        cfg = O.make_config(80, 50, 0, 1, 0)
        base, near = oracle_frames(s, O.make_camera(pos=cam, fov_deg=65.0), cfg)
        u = sr.uniforms(sr.camera(cam, 65.0), 80, 50, 0, 1, 0, num_nodes=int(s.info.n_nodes),
                        num_stars=int(s.info.n_stars), light_pos=_light4(s))
        fr = engine.render(BASE + w, u, path=path, aux=True)
        rep = compare(fr, base, near)
        print(f"demo {w} path {path}:", rep)
        assert (fr.rgb != 0).all()
        assert rep.hit_match_nongrazing == 1.0 and rep.lam_max_rel <= 1e-5 and rep.tau_max_rel <= 1e-5
        assert rep.rgb_max_unmasked <= 1


def _lit_fraction(engine, s, tau):
    cam0 = s.initial_camera
    pos = (cam0[0] + tau, cam0[1], cam0[2], cam0[3])
    kw = dict(num_nodes=int(s.info.n_nodes), num_stars=int(s.info.n_stars), light_pos=_light4(s))
    plain = engine.render(BASE, sr.uniforms(sr.camera(pos, 65.0), 160, 100, 0, 1, 0, **kw)).rgb
    lit = engine.render(BASE, sr.uniforms(sr.camera(pos, 65.0), 160, 100, 0, 1, 0,
                                          flashes=[(cam0, 0.8, 2.5, (1.0, 0.9, 0.7))], **kw)).rgb
    return float((plain != lit).mean())


def test_player_flash_visible_after_round_trip(engine, demos):
    s = demos[O.DEMO_TWIN_PARADOX]
    at_10 = _lit_fraction(engine, s, 10.0)
    print("engine: flash lit", at_10)
    assert at_10 > 0.01
    assert _lit_fraction(engine, s, 120.0) == 0.0
