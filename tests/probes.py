"""The reference's end-to-end physics probes (src/scene.rs:785-1053) over a ray-query callable, so the
same probes run on the oracle (Bvh4D::trace restated, CPU) and on the engine (sr_trace_rays, GPU).

A tracer takes rays (n x 10: origin t, x, y, z, direction, t_min, t_max) and returns a dict of
arrays: found, lam, tau, event (n x 4), id. Ray set-up follows the reference in f32 (numpy float32:
each operation rounded as Rust's f32 code rounds it; sin / cos only enter the Penrose probe, whose
bar is 1.5%). Each probe asserts the reference's own bar and returns what it measured.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

f32 = np.float32
MISS = 0xFFFFFFFF
Z = (f32(0), f32(0), f32(0), f32(1))  # the +z spatial ray the probes aim with (t, x, y, z)


def oracle_tracer(scene):
    def trace(rays):
        out = scene.trace(rays)
        return dict(found=out[:, 0] > 0, lam=out[:, 3], tau=out[:, 4], event=out[:, 5:9], id=out[:, 2])
    return trace


def engine_tracer(engine, idx):
    def trace(rays):
        h = engine.trace_rays(idx, rays)
        return dict(found=h["id"] != MISS, lam=h["lambda_"].astype(np.float64), tau=h["proper_time"].astype(np.float64),
                    event=np.array(h["event"], np.float64), id=h["id"].astype(np.float64))
    return trace


def ray(origin, direction, t_min, t_max):
    return np.array([*[float(x) for x in origin], *[float(f32(x)) for x in direction], float(f32(t_min)),
                     float(f32(t_max))], np.float64)


def normalized(v):
    """Vec3::normalized (minkowski.rs:47-54): v * (1 / sqrt((x x + y y) + z z))."""
    v = np.asarray(v, f32)
    n = np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2], dtype=f32)
    return v * (f32(1) / n) if n > f32(1e-12) else np.zeros(3, f32)


def cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], f32)


def spatial_to_world(E, l):
    """Tetrad::local_spatial_to_world: e1 l.x + e2 l.y + e3 l.z (rows of E are e0..e3)."""
    return E[1] * l[0] + E[2] * l[1] + E[3] * l[2]


def past_light_ray(E, l):
    """Tetrad::past_light_ray_direction (minkowski.rs:564-567): -e0 + e1 n.x + e2 n.y + e3 n.z."""
    n = normalized(l)
    return -E[0] + E[1] * n[0] + E[2] * n[1] + E[3] * n[2]


REST = np.eye(4, dtype=f32)


def twin_aging(trace):
    """test_twin_paradox_differential_clock_aging (scene.rs:785-813)."""
    r = trace(np.stack([ray((15.0, -1.2, -1.05, 0.0), Z, 0.1, 20.0), ray((15.0, 1.4, -1.05, 0.0), Z, 0.1, 20.0)]))
    assert r["found"].all(), "should hit both twins"
    home, trav = r["tau"]
    assert abs(home - 29.0) < 0.05, f"home proper_time = {home}"
    assert trav < home - 7.0, f"traveler {trav} should be >7 s younger than home {home}"
    return home, trav


def barn_and_pole(trace):
    """test_barn_and_pole_world_slice_vs_camera_slice (scene.rs:816-868)."""
    r = trace(np.stack([ray((0.0, -1.5, -0.85, 0.0), Z, 0.1, 10.0), ray((0.0, 1.5, -0.85, 0.0), Z, 0.1, 10.0)]))
    assert r["found"].all(), "should hit rear and front of the pole in the world slice"
    measured = r["tau"][0] - r["tau"][1]
    expected = float((f32(1) / np.sqrt(f32(1) - f32(0.85) * f32(0.85), dtype=f32)) * f32(0.85) * f32(3.0))
    assert abs(measured - expected) < 0.05, f"world slice delta_tau = {measured}, expected = {expected}"
    E = O.tetrad_from_beta((0.85, 0.0, 0.0))
    d_rear = spatial_to_world(E, normalized((-3.5, 0.0, 6.0)))
    d_front = spatial_to_world(E, normalized((3.5, 0.0, 6.0)))
    o = (0.0, 0.0, -0.85, 0.0)
    c = trace(np.stack([ray(o, d_rear, 0.1, 20.0), ray(o, d_front, 0.1, 20.0)]))
    assert c["found"].all(), "should hit the pole at rest-frame x' = -3.5 and +3.5 in the camera slice"
    assert abs(c["tau"][0] - c["tau"][1]) < 0.02, f"camera slice taus {c['tau']} should be identical"
    return measured, expected, tuple(c["tau"])


def train_sync(trace):
    """test_einstein_train_all_wagons_visible_and_synced (scene.rs:871-903): every wagon at every
    probed lab time shows tau = gamma (t - beta x)."""
    beta = f32(0.80)
    gamma = f32(1) / np.sqrt(f32(1) - beta * beta, dtype=f32)
    rays, expect = [], []
    for t in (f32(-14), f32(-7), f32(0), f32(7), f32(14)):
        for i in range(-3, 4):
            x_rest = f32(i) * f32(2.6)
            x_lab = x_rest / gamma + beta * t
            rays.append(ray((t, x_lab, 1.05, 0.0), Z, 0.1, 15.0))
            expect.append(float(gamma * (t - beta * x_lab)))
    r = trace(np.stack(rays))
    assert r["found"].all(), f"wagons clipped: {np.nonzero(~r['found'])[0]}"
    err = np.abs(r["tau"] - np.array(expect))
    assert err.max() < 0.05, f"max |tau - gamma (t - beta x)| = {err.max()}"
    return float(err.max())


def loop_continuity(trace, window):
    """test_loop_boundary_past_light_cone_continuity (scene.rs:906-949): the past light cone at
    t_min hits the previous loop's pole where the one at t_max hits this loop's."""
    cam = np.array((0.0, -0.85, -3.2), f32)
    target = np.array((2.0, -0.85, 6.0), f32)
    d = past_light_ray(REST, target - cam)
    t_min, t_max = window
    r = trace(np.stack([ray((t_max, *cam), d, 0.1, 30.0), ray((t_min, *cam), d, 0.1, 30.0)]))
    assert r["found"].all(), "should hit the pole at both ends of the loop"
    ds = float(np.linalg.norm(r["event"][0, 1:] - r["event"][1, 1:]))
    dt = abs(r["tau"][0] - r["tau"][1])
    assert ds < 1e-3, f"spatial hit position jumped across the loop wrap by {ds}"
    assert dt < 1e-2, f"proper time jumped across the loop wrap by {dt}"
    return ds, dt


def penrose_circularity(trace):
    """test_penrose_sphere_circular_silhouette (scene.rs:985-1053): a sphere moving at 0.8 c casts
    a circular silhouette (angular radius within 1.5% over 8 azimuths), by bisection of hit / miss."""
    beta = np.array((0.80, 0.0, 0.0), f32)
    pos = np.array((0.0, 0.0, 8.0), f32)
    a = f32(1) - (beta[0] * beta[0] + beta[1] * beta[1] + beta[2] * beta[2])
    b = f32(-2) * (pos[0] * beta[0] + pos[1] * beta[1] + pos[2] * beta[2])
    c = -(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2])
    t_ret = (-b - np.sqrt(b * b - f32(4) * a * c, dtype=f32)) / (f32(2) * a)
    retarded = normalized(pos + beta * t_ret)
    up = np.array((0.0, 1.0, 0.0), f32)
    u_perp = normalized(cross(up, retarded))

    def find_edge(center, radial):
        lo, hi = f32(0), f32(0.45)
        for _ in range(20):
            mid = f32(0.5) * (lo + hi)
            d = center * np.cos(mid, dtype=f32) + radial * np.sin(mid, dtype=f32)
            hit = trace(ray((0.0, 0.0, 0.0, 0.0), past_light_ray(REST, d), 0.1, 30.0)[None])["found"][0]
            if hit:
                lo = mid
            else:
                hi = mid
        return f32(0.5) * (lo + hi)

    r_plus, r_minus = find_edge(retarded, u_perp), find_edge(retarded, -u_perp)
    shift = f32(0.5) * (r_plus - r_minus)
    center = normalized(retarded * np.cos(shift, dtype=f32) + u_perp * np.sin(shift, dtype=f32))
    u_c = normalized(cross(up, center))
    v_c = normalized(cross(center, u_c))
    radii = []
    for k in range(8):
        phi = f32(k) * f32(2 * np.pi) / f32(8)
        radii.append(find_edge(center, u_c * np.cos(phi, dtype=f32) + v_c * np.sin(phi, dtype=f32)))
    radii = np.array(radii, np.float64)
    mean = radii.mean()
    dev = np.abs(radii - mean) / mean
    assert dev.max() < 0.015, f"silhouette radii {radii} deviate {dev.max()} from their mean {mean}"
    return radii, float(dev.max())


def checked_tracer(engine_trace, oracle_trace, log):
    """The engine's tracer, holding every call's hits to the oracle's on the same rays: the same
    simplex, lambda and proper time bit for bit (both are f32 on the reference's traversal)."""
    def trace(rays):
        e, o = engine_trace(rays), oracle_trace(rays)
        assert (e["found"] == o["found"]).all(), "hit / miss differs from the oracle"
        f = e["found"]
        assert (e["id"][f] == o["id"][f]).all(), "hit simplex differs from the oracle"
        assert (e["lam"][f] == o["lam"][f]).all() and (e["tau"][f] == o["tau"][f]).all(), "lambda / tau differ"
        log.append(len(rays))
        return e
    return trace
