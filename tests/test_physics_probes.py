"""The reference's end-to-end known answers, on the CPU: its demo scenes restated in the oracle
(oracle/oracle_demo.hpp) must pass the reference's own physics probes with the reference's own
bars (src/scene.rs:733-1053), and the caller-side FrameDynamics helpers of the engine library
(host code, no device) must pass src/renderer.rs:1171-1229.

The same probes run on the engine in test_physics_probes_gpu.py."""
import ctypes as C

import numpy as np
import pytest

import probes as P
from oracle import oracle as O


@pytest.fixture(scope="module")
def demos():
    return {w: O.Scene.demo(w) for w in range(5)}


def test_twin_paradox_differential_clock_aging(demos):
    home, trav = P.twin_aging(P.oracle_tracer(demos[O.DEMO_TWIN_PARADOX]))
    print("home", home, "traveler", trav)


def test_barn_and_pole_world_slice_vs_camera_slice(demos):
    print(P.barn_and_pole(P.oracle_tracer(demos[O.DEMO_BARN_AND_POLE])))


def test_einstein_train_all_wagons_visible_and_synced(demos):
    print("max tau error", P.train_sync(P.oracle_tracer(demos[O.DEMO_EINSTEIN_TRAIN])))


def test_loop_boundary_past_light_cone_continuity(demos):
    s = demos[O.DEMO_BARN_AND_POLE]
    print(P.loop_continuity(P.oracle_tracer(s), s.window))


def test_penrose_sphere_circular_silhouette():
    radii, dev = P.penrose_circularity(P.oracle_tracer(O.Scene.demo(O.PENROSE_SPHERE)))
    print("radii", radii, "max deviation", dev)


def test_light_clock_subluminal_exact_speed_c():
    """test_light_clock_subluminal_exact_speed_c (scene.rs:952-982)."""
    m = O.material(5)
    assert m["pattern"] == 2  # SurfacePattern::LightClock
    L = np.float32(m["cavity_length"])
    assert abs(L - 1.0) < 1e-6
    f = O.light_clock_bounce_fraction
    assert abs(f(0.0, L) - 0.0) < 1e-6
    assert abs(f(0.5, L) - 0.5) < 1e-6
    assert abs(f(1.0, L) - 1.0) < 1e-6
    assert abs(f(2.0, L) - 0.0) < 1e-6
    beta = np.float32(0.80)
    gamma = np.float32(1) / np.sqrt(np.float32(1) - beta * beta, dtype=np.float32)
    t_half = gamma * L
    assert abs(f(float(t_half / gamma), L) - 1.0) < 1e-5
    path = np.sqrt(L * L + (beta * t_half) ** 2, dtype=np.float32)
    assert abs(path / t_half - 1.0) < 1e-5


def test_all_five_paradox_scenes_render(demos):
    """test_all_five_paradox_scenes_render (scene.rs:733-754): every static demo scene renders at
    80x50 (shaded, Lorentz-invariant shadows, past light cone) with no black pixel. The sixth demo
    (RelativisticBilliards) is a dynamic-mode world, outside this path."""
    for w, s in demos.items():
        r = O.render(s, O.make_camera(pos=s.initial_camera, fov_deg=65.0), O.make_config(80, 50, 0, 1, 0), aux=False)
        assert (r.rgb != 0).all(), f"demo {w} has black pixels"


def _flash_lit_fraction(scene, tau, width=160, height=100):
    cam0 = scene.initial_camera
    at = cam0
    pos = (cam0[0] + tau, cam0[1], cam0[2], cam0[3])  # cam.position += e0 * tau (rest tetrad)
    cam = O.make_camera(pos=pos, fov_deg=65.0)
    cfg = O.make_config(width, height, 0, 1, 0)
    plain = O.render(scene, cam, cfg, aux=False).rgb
    dyn = O.DynamicsSpec(flashes=[(at, 0.8, 2.5, (1.0, 0.9, 0.7))])  # FrameDynamics::emit_flash
    lit = O.render(scene, cam, cfg, dyn, aux=False).rgb
    return float((plain != lit).mean())


def test_player_flash_visible_after_round_trip(demos):
    """test_player_flash_visible_after_round_trip (scene.rs:757-782): a flash from the camera lights
    the twins' clocks 5 ls away after 10 s (out and back), and nothing after 120 s."""
    s = demos[O.DEMO_TWIN_PARADOX]
    at_10 = _flash_lit_fraction(s, 10.0)
    assert at_10 > 0.01, f"flash lit only {at_10 * 100:.2f}% of pixels after 10 s"
    assert _flash_lit_fraction(s, 120.0) == 0.0


def test_flash_slots_evict_retire_and_shift():
    """renderer.rs:1171-1189 against the engine library's caller-side flash list."""
    from specrel_b200 import _lib as L
    lib = L.lib()
    fl = (L.Flash * L.SR_MAX_FLASHES)()
    n = C.c_uint32(0)
    for i in range(L.SR_MAX_FLASHES + 3):
        assert lib.sr_flash_emit(fl, C.byref(n), (C.c_float * 4)(float(i), 0.0, 0.0, 0.0), 0) == L.SR_OK
    assert n.value == L.SR_MAX_FLASHES
    assert fl[0].at[0] == 3.0, "oldest flashes are evicted first"
    assert (fl[0].width, fl[0].intensity, tuple(fl[0].color)) == (np.float32(0.8), 2.5, tuple(np.float32([1.0, 0.9, 0.7])))
    assert lib.sr_flashes_shift_time(fl, n.value, -100.0) == L.SR_OK
    assert fl[0].at[0] == -97.0
    # Flashes now sit at t = -97 ..= -82; at now = 110 only those with t > -90 survive.
    assert lib.sr_flashes_retire(fl, C.byref(n), 110.0) == L.SR_OK
    assert all(110.0 - fl[i].at[0] < 200.0 for i in range(n.value))
    assert n.value == 8


def test_prophecy_delta_steps_are_clamped():
    """renderer.rs:1214-1229 against the engine library's RenderConfig helper."""
    from specrel_b200 import _lib as L
    lib = L.lib()
    cfg = L.RenderConfig(1, 1, 0, 0, 3, 3.5)
    lib.sr_config_step_prophecy_delta(C.byref(cfg), 2.0)
    assert cfg.prophecy_delta == np.float32(3.5) + 2.0 * np.float32(0.5)
    lib.sr_config_step_prophecy_delta(C.byref(cfg), -1000.0)
    assert cfg.prophecy_delta == np.float32(0.5)
    lib.sr_config_step_prophecy_delta(C.byref(cfg), 1000.0)
    assert cfg.prophecy_delta == np.float32(20.0)
