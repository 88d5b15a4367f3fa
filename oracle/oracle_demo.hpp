// TEST INFRASTRUCTURE ONLY — part of the CPU oracle that the parity tests use as the checker.
// Nothing in the shipped library includes, links or calls this file.
//
// The reference's demo scenes, restated so that its end-to-end physics probes (scene.rs:733-1053:
// twin aging, barn and pole, Einstein's train, loop continuity, light clock, Penrose silhouette,
// render and flash visibility) can be run against the oracle and, through the packed arrays,
// against the engine:
//   src/mesh4d.rs:508-563   Mesh3D::uv_sphere
//   src/mesh4d.rs:566-611   Mesh3D::ground_grid
//   src/mesh4d.rs:1056-1087 sync_proper_time_at
//   src/star.rs:290-318     starfield (the demo scenes' backdrop, scene.rs:177-179)
//   src/scene.rs:92-101     DemoScene::initial_camera_pos
//   src/scene.rs:124-139    twin_traveler_x_and_vx
//   src/scene.rs:141-150    for_periodic_copies
//   src/scene.rs:283-720    build_twin_paradox, build_barn_and_pole, build_terrell_penrose_street,
//                           build_einstein_train, build_carousel
// Arithmetic follows the reference's types: f32 where it computes in f32 (the scalar type T of the
// oracle), f64 where it computes in f64 (worldline position functions).
#pragma once
#include <cmath>
#include <cstdint>
#include <functional>
#include <vector>

#include "oracle_scenes.hpp"

namespace orc {

// Mesh3D::uv_sphere (mesh4d.rs:508-563).
template <class T> Mesh3D<T> uv_sphere(T radius, size_t lat_steps, size_t lon_steps) {
    Mesh3D<T> m;
    for (size_t i = 0; i <= lat_steps; ++i) {
        T v = (T)i / (T)lat_steps;
        T theta = v * C<T>::PI;
        T sin_t = m_sin(theta), cos_t = m_cos(theta);
        for (size_t j = 0; j <= lon_steps; ++j) {
            T u = (T)j / (T)lon_steps;
            T phi = u * C<T>::TAU;
            T sin_p = m_sin(phi), cos_p = m_cos(phi);
            m.vertices.push_back(V3<T>(radius * sin_t * cos_p, radius * cos_t, radius * sin_t * sin_p));
        }
    }
    const size_t stride = lon_steps + 1;
    for (size_t i = 0; i < lat_steps; ++i)
        for (size_t j = 0; j < lon_steps; ++j) {
            const uint32_t i00 = (uint32_t)(i * stride + j), i10 = i00 + 1, i01 = (uint32_t)((i + 1) * stride + j),
                           i11 = i01 + 1;
            T u0 = (T)j / (T)lon_steps * T(4), u1 = (T)(j + 1) / (T)lon_steps * T(4);
            T v0 = (T)i / (T)lat_steps * T(2), v1 = (T)(i + 1) / (T)lat_steps * T(2);
            if (i > 0) {
                V3<T> n = (m.vertices[i00] + m.vertices[i10] + m.vertices[i11]).normalized();
                m.triangles.push_back({{i00, i11, i10}, {{{u0, v0}, {u1, v1}, {u1, v0}}}, n});
            }
            if (i + 1 < lat_steps) {
                V3<T> n = (m.vertices[i00] + m.vertices[i01] + m.vertices[i11]).normalized();
                m.triangles.push_back({{i00, i01, i11}, {{{u0, v0}, {u0, v1}, {u1, v1}}}, n});
            }
        }
    return m;
}

// Mesh3D::ground_grid (mesh4d.rs:566-611): the XZ plane at height y, uv = (x, z).
template <class T> Mesh3D<T> ground_grid(T half_x, T half_z, T y, size_t divs_x, size_t divs_z) {
    Mesh3D<T> m;
    for (size_t iz = 0; iz <= divs_z; ++iz) {
        T fz = (T)iz / (T)divs_z;
        T z = -half_z + fz * (T(2) * half_z);
        for (size_t ix = 0; ix <= divs_x; ++ix) {
            T fx = (T)ix / (T)divs_x;
            T x = -half_x + fx * (T(2) * half_x);
            m.vertices.push_back(V3<T>(x, y, z));
        }
    }
    const size_t stride = divs_x + 1;
    const V3<T> normal(T(0), T(1), T(0));
    for (size_t iz = 0; iz < divs_z; ++iz)
        for (size_t ix = 0; ix < divs_x; ++ix) {
            const uint32_t i00 = (uint32_t)(iz * stride + ix), i10 = i00 + 1, i01 = (uint32_t)((iz + 1) * stride + ix),
                           i11 = i01 + 1;
            const V3<T> p00 = m.vertices[i00], p10 = m.vertices[i10], p01 = m.vertices[i01], p11 = m.vertices[i11];
            m.triangles.push_back({{i00, i01, i11}, {{{p00.x, p00.z}, {p01.x, p01.z}, {p11.x, p11.z}}}, normal});
            m.triangles.push_back({{i00, i11, i10}, {{{p00.x, p00.z}, {p11.x, p11.z}, {p10.x, p10.z}}}, normal});
        }
    return m;
}

// sync_proper_time_at (mesh4d.rs:1056-1087): proper time and phi shifted to 0 at lab time t_sync
// (linear interpolation between the samples around it, clamped to the ends).
template <class T> void sync_proper_time_at(std::vector<WorldlineSample<T>>& s, T t_sync) {
    if (s.empty()) return;
    T tau = s[0].proper_time;
    V3<T> phi = s[0].phi;
    if (t_sync <= s[0].center.t) {
        tau = s[0].proper_time;
        phi = s[0].phi;
    } else if (t_sync >= s.back().center.t) {
        tau = s.back().proper_time;
        phi = s.back().phi;
    } else {
        for (size_t k = 0; k + 1 < s.size(); ++k) {
            const auto &s0 = s[k], &s1 = s[k + 1];
            if (t_sync >= s0.center.t && t_sync <= s1.center.t) {
                T dt = fmax_(s1.center.t - s0.center.t, T(1e-6));
                T frac = (t_sync - s0.center.t) / dt;
                tau = s0.proper_time + frac * (s1.proper_time - s0.proper_time);
                phi = s0.phi + (s1.phi - s0.phi) * frac;
                break;
            }
        }
    }
    for (auto& x : s) {
        x.proper_time -= tau;
        x.phi -= phi;
    }
}

// starfield (star.rs:290-318): `count` stars around `center` at radii [r_min, r_max] from a
// PCG-style hash of `seed`; every seventh star (i % 7 == 3) moving at 0.6 c.
template <class T> std::vector<PointStar<T>> starfield(const V3<T>& center, size_t count, T r_min, T r_max, uint32_t seed) {
    uint32_t state = seed * 747796405u + 2891336453u;
    auto next = [&]() -> T {
        state = state * 747796405u + 2891336453u;
        uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
        return (T)((word >> 22) ^ word) / (T)4294967295u;
    };
    std::vector<PointStar<T>> out;
    for (size_t i = 0; i < count; ++i) {
        T z = next() * T(1.7) - T(0.7);
        T phi = next() * C<T>::TAU;
        T rho = m_sqrt(fmax_(T(1) - z * z, T(0)));
        V3<T> dir(rho * m_cos(phi), z, rho * m_sin(phi));
        T r = r_min + (r_max - r_min) * next();
        T a0 = next();
        T temperature = T(2800) + T(14000) * a0 * next();
        T intensity = r * r * T(2e-4) * m_powf(T(10), T(2) * next());
        V3<T> beta;
        if (i % 7 == 3) {
            T a = next() * C<T>::TAU;
            T bx = m_cos(a);
            T by = T(0.2) * (next() - T(0.5));
            beta = V3<T>(bx, by, m_sin(a)) * T(0.6);
        }
        out.push_back(PointStar<T>::moving(center + dir * r, beta, temperature, intensity));
    }
    return out;
}

// twin_traveler_x_and_vx (scene.rs:124-139): rest at x = 1.4 outside [-14, 14], a raised-cosine
// excursion inside it (peak 0.9425 c). f64.
inline void twin_traveler_x_and_vx(double t_rel, double* x, double* vx) {
    const double x_start = 1.4, t_dep = -14.0, t_ret = 14.0;
    if (t_rel <= t_dep || t_rel >= t_ret) {
        *x = x_start;
        *vx = 0.0;
        return;
    }
    const double omega = 6.283185307179586 / (t_ret - t_dep), amp = 4.2;
    const double phase = omega * (t_rel - t_dep);
    *x = x_start + amp * (1.0 - std::cos(phase));
    *vx = amp * omega * std::sin(phase);
}

// PENROSE_SPHERE is not a demo scene: it is the scene test_penrose_sphere_circular_silhouette builds
// for itself (scene.rs:985-996), a uv sphere of radius 1.2 moving at 0.8 c, with no ground, light
// or backdrop stars.
enum DemoScene : uint32_t {
    TWIN_PARADOX = 0, BARN_AND_POLE = 1, TERRELL_PENROSE_STREET = 2, EINSTEIN_TRAIN = 3, CAROUSEL = 4, PENROSE_SPHERE = 5
};

template <class T> struct DemoOut {
    SynthOut<T> s;
    T t_min = 0, t_max = 0;
};

template <class T> DemoOut<T> build_demo(uint32_t which) {
    DemoOut<T> out;
    std::vector<Simplex<T>> all;
    auto tube = [&](const Mesh3D<T>& mesh, const std::vector<WorldlineSample<T>>& wl, uint32_t mat) {
        out.s.rindler_ok &= extend_worldtube_simplices<T>(all, mesh, wl, (const T*)nullptr, mat);
    };
    auto inertial = [](T x, T y, T z, const V3<T>& beta, T t0, T t1, size_t steps) {
        return sample_inertial_worldline<T>(V3<T>(x, y, z), beta, t0, t1, steps);
    };
    auto accelerated = [&](std::function<Pos3d(double)> f, T t0, T t1, size_t steps) {
        bool sl = false;
        auto w = sample_accelerated_worldline<T>(f, t0, t1, steps, &sl);
        out.s.superluminal |= sl;
        return w;
    };
    auto periodic = [](T t_loop, int k0, int k1, const std::function<void(T)>& copy) {  // scene.rs:141-150
        for (int k = k0; k <= k1; ++k) copy((T)k * t_loop);
    };
    const V3<T> rest;
    V3<T> light;
    double cam[4] = {0, 0, 0, 0};
    if (which == TWIN_PARADOX) {  // scene.rs:283-381
        out.t_min = T(-18);
        out.t_max = T(34);
        const T t_loop = out.t_max - out.t_min, t_sync_base = T(-14);
        tube(ground_grid<T>(T(22), T(24), T(-2.2), 4, 4), inertial(0, 0, 0, rest, T(-160), T(120), 1), 0);
        const Mesh3D<T> twin = Mesh3D<T>::cube(V3<T>(T(1.15), T(1.15), T(1.15)));
        const Mesh3D<T> pillar = Mesh3D<T>::cube(V3<T>(T(0.55), T(0.625), T(0.55)));
        const Mesh3D<T> marker = Mesh3D<T>::cube(V3<T>(T(0.6), T(0.6), T(0.6)));
        periodic(t_loop, -2, 1, [&](T t_off) {
            const T seg0 = out.t_min + t_off, seg1 = out.t_max + t_off, t_sync = t_sync_base + t_off;
            auto home = inertial(T(-1.2), T(-1.05), T(6.0), rest, seg0, seg1, 2);
            sync_proper_time_at(home, t_sync);
            tube(twin, home, 1);
            auto home_lc = inertial(T(-3.2), T(-1.575), T(6.0), rest, seg0, seg1, 2);
            sync_proper_time_at(home_lc, t_sync);
            tube(pillar, home_lc, 5);
            const double off = (double)t_off;
            auto trav = accelerated([off](double t) { double x, vx; twin_traveler_x_and_vx(t - off, &x, &vx); return Pos3d{x, -1.05, 6.0}; },
                                    seg0, seg1, 120);
            sync_proper_time_at(trav, t_sync);
            tube(twin, trav, 2);
            auto trav_lc = accelerated([off](double t) { double x, vx; twin_traveler_x_and_vx(t - off, &x, &vx); return Pos3d{x, 0.725, 6.0}; },
                                       seg0, seg1, 120);
            sync_proper_time_at(trav_lc, t_sync);
            tube(pillar, trav_lc, 5);
            auto mk = inertial(T(9.2), T(-1.6), T(7.8), rest, seg0, seg1, 2);
            sync_proper_time_at(mk, t_sync);
            tube(marker, mk, 3);
        });
        light = V3<T>(T(2.0), T(6.5), T(2.0));
        cam[0] = -15.0; cam[1] = 2.2; cam[2] = 0.0; cam[3] = -3.5;
    } else if (which == BARN_AND_POLE) {  // scene.rs:383-458
        out.t_min = T(-12);
        out.t_max = T(12);
        const T t_loop = out.t_max - out.t_min;
        tube(ground_grid<T>(T(22), T(22), T(-2.2), 4, 4), inertial(0, 0, 0, rest, T(-140), T(140), 1), 0);
        const Mesh3D<T> door = Mesh3D<T>::cube(V3<T>(T(0.35), T(1.5), T(0.35)));
        for (T x : {T(-2.85), T(2.85)}) tube(door, inertial(x, T(-0.7), T(5.2), rest, T(-140), T(140), 1), 1);
        tube(Mesh3D<T>::cube(V3<T>(T(3.2), T(0.8), T(0.6))), inertial(T(0), T(1.6), T(5.8), rest, T(-140), T(140), 1), 1);
        tube(Mesh3D<T>::cube(V3<T>(T(2.5), T(1.5), T(0.25))), inertial(T(0), T(-0.7), T(7.4), rest, T(-140), T(140), 1), 6);
        const Mesh3D<T> pole = Mesh3D<T>::cube(V3<T>(T(4.0), T(0.55), T(0.45)));
        const V3<T> beta(T(0.85), T(0), T(0));
        periodic(t_loop, -2, 1, [&](T t_off) {
            const V3<T> p0 = V3<T>(T(0), T(-0.85), T(6.0)) - beta * t_off;
            auto wl = sample_inertial_worldline<T>(p0, beta, t_off - T(55), t_off + T(55), 12);
            sync_proper_time_at(wl, t_off);
            tube(pole, wl, 2);
        });
        light = V3<T>(T(0.0), T(6.0), T(1.5));
        cam[0] = -4.5; cam[1] = 0.0; cam[2] = 0.1; cam[3] = -3.2;
    } else if (which == TERRELL_PENROSE_STREET) {  // scene.rs:460-574
        out.t_min = T(-14);
        out.t_max = T(14);
        const T t_loop = out.t_max - out.t_min;
        tube(ground_grid<T>(T(20), T(28), T(-2.2), 4, 6), inertial(0, 0, 0, rest, T(-140), T(140), 1), 0);
        const Mesh3D<T> pillar = Mesh3D<T>::cube(V3<T>(T(0.95), T(0.95), T(0.95)));
        const Mesh3D<T> lc = Mesh3D<T>::cube(V3<T>(T(0.65), T(0.625), T(0.65)));
        for (int iz = -3; iz <= 3; ++iz) {
            const T z = (T)iz * T(5.0);
            for (T x : {T(-4.2), T(4.2)}) {
                if (iz == 0) tube(lc, inertial(x, T(-1.575), z, rest, T(-140), T(140), 1), 5);
                else tube(pillar, inertial(x, T(-1.25), z, rest, T(-140), T(140), 1), 1);
            }
        }
        const Mesh3D<T> flyer = Mesh3D<T>::cube(V3<T>(T(1.05), T(1.05), T(1.05)));
        const V3<T> beta_flyer(T(0.85), T(0), T(0));
        const Mesh3D<T> sphere = uv_sphere<T>(T(1.05), 10, 16);
        const V3<T> beta_sphere(T(0), T(0), T(-0.86));
        periodic(t_loop, -2, 1, [&](T t_off) {
            auto fw = sample_inertial_worldline<T>(V3<T>(T(0), T(-0.75), T(4.5)) - beta_flyer * t_off, beta_flyer,
                                                   t_off - T(55), t_off + T(55), 10);
            sync_proper_time_at(fw, t_off);
            tube(flyer, fw, 2);
            auto sw = sample_inertial_worldline<T>(V3<T>(T(-1.8), T(0.6), T(5.0)) - beta_sphere * t_off, beta_sphere,
                                                   t_off - T(55), t_off + T(55), 10);
            sync_proper_time_at(sw, t_off);
            tube(sphere, sw, 6);
        });
        const double omega0 = 6.283185307179586 / (double)t_loop;
        tube(Mesh3D<T>::cube(V3<T>(T(0.95), T(0.95), T(0.95))),
             accelerated([omega0](double t) { return Pos3d{3.6 * std::sin(omega0 * t), 1.1, 8.5}; }, T(-110), T(70), 260), 3);
        tube(Mesh3D<T>::cube(V3<T>(T(0.75), T(0.75), T(0.75))),
             accelerated([omega0](double t) { return Pos3d{1.5 + 3.2 * std::cos(omega0 * t), 0.5, 11.5 + 3.2 * std::sin(omega0 * t)}; },
                         T(-110), T(70), 260),
             4);
        light = V3<T>(T(0.0), T(6.5), T(4.0));
        cam[0] = 0.0; cam[1] = 0.0; cam[2] = 0.0; cam[3] = -7.5;
    } else if (which == EINSTEIN_TRAIN) {  // scene.rs:576-646
        out.t_min = T(-14);
        out.t_max = T(14);
        const T t_loop = out.t_max - out.t_min;
        tube(ground_grid<T>(T(24), T(22), T(-2.2), 4, 4), inertial(0, 0, 0, rest, T(-140), T(140), 1), 0);
        const Mesh3D<T> clock = Mesh3D<T>::cube(V3<T>(T(0.95), T(0.95), T(0.95)));
        for (int i = -3; i <= 3; ++i) tube(clock, inertial((T)i * T(2.6), T(-1.15), T(6.8), rest, T(-140), T(140), 1), 1);
        tube(Mesh3D<T>::cube(V3<T>(T(0.55), T(0.625), T(0.55))), inertial(T(0), T(-1.575), T(5.1), rest, T(-140), T(140), 1), 5);
        const V3<T> beta(T(0.80), T(0), T(0));
        const T gamma = T(1) / m_sqrt(T(1) - beta.x * beta.x);
        periodic(t_loop, -2, 1, [&](T t_off) {
            for (int i = -3; i <= 3; ++i) {
                const T x_rest = (T)i * T(2.6);
                const V3<T> p0 = V3<T>(x_rest / gamma, T(1.05), T(6.8)) - beta * t_off;
                const T t_sync = t_off + gamma * beta.x * x_rest;
                auto wl = sample_inertial_worldline<T>(p0, beta, t_off - T(60), t_off + T(60), 10);
                sync_proper_time_at(wl, t_sync);
                tube(clock, wl, 2);
            }
        });
        light = V3<T>(T(0.0), T(6.5), T(2.0));
        cam[0] = -3.0; cam[1] = 0.0; cam[2] = 0.0; cam[3] = -4.5;
    } else if (which == PENROSE_SPHERE) {  // scene.rs:989-996
        out.t_min = T(-40);
        out.t_max = T(40);
        tube(uv_sphere<T>(T(1.2), 24, 36),
             sample_inertial_worldline<T>(V3<T>(T(0), T(0), T(8)), V3<T>(T(0.8), T(0), T(0)), T(-40), T(40), 4), 0);
        auto& sc = out.s.scene;
        sc.materials = common_materials<T>();
        sc.light_pos = V3<T>(T(0), T(50), T(0));
        sc.finish_stars();
        sc.bvh = Bvh<T>::build(std::move(all));
        return out;
    } else {  // CAROUSEL, scene.rs:648-720
        out.t_min = T(-24);
        out.t_max = T(24);
        const T t_loop = out.t_max - out.t_min, t_sync = T(-20);
        tube(ground_grid<T>(T(22), T(24), T(-2.2), 4, 4), inertial(0, 0, 0, rest, T(-140), T(120), 1), 0);
        auto master = inertial(T(0), T(-0.7), T(8.0), rest, T(-110), T(70), 2);
        sync_proper_time_at(master, t_sync);
        tube(Mesh3D<T>::cube(V3<T>(T(1.05), T(1.05), T(1.05))), master, 1);
        auto lcw = inertial(T(0), T(0.975), T(8.0), rest, T(-110), T(70), 2);
        sync_proper_time_at(lcw, t_sync);
        tube(Mesh3D<T>::cube(V3<T>(T(0.55), T(0.625), T(0.55))), lcw, 5);
        const Mesh3D<T> orbiter = Mesh3D<T>::cube(V3<T>(T(0.62), T(0.62), T(0.62)));
        const double omega = 2.0 * 6.283185307179586 / (double)t_loop, radius = 0.80 / omega, ts = (double)t_sync;
        for (int k = 0; k < 6; ++k) {
            const double phase0 = (double)k * 6.283185307179586 / 6.0;
            auto wl = accelerated(
                [=](double t) {
                    const double angle = omega * (t - ts) + phase0;
                    return Pos3d{radius * std::cos(angle), -0.6 + 0.25 * std::sin(2.0 * angle), 8.0 + radius * std::sin(angle)};
                },
                T(-110), T(70), 320);
            sync_proper_time_at(wl, t_sync);
            tube(orbiter, wl, k % 2 == 0 ? 2u : 3u);
        }
        light = V3<T>(T(0.0), T(6.8), T(3.0));
        cam[0] = -18.0; cam[1] = 0.0; cam[2] = 0.8; cam[3] = -2.5;
    }
    auto& sc = out.s.scene;
    sc.materials = common_materials<T>();
    sc.light_pos = light;
    sc.stars = starfield<T>(V3<T>(), 90, T(60), T(170), 7);  // Scene4D::backdrop_stars (scene.rs:177-179)
    sc.finish_stars();
    sc.bvh = Bvh<T>::build(std::move(all));
    for (int k = 0; k < 4; ++k) out.s.cam_pos[k] = cam[k];
    return out;
}

}  // namespace orc
