// TEST INFRASTRUCTURE ONLY — part of the CPU oracle used by the parity tests as the checker.
//
// The seeded synthetic workloads (the five benchmark configurations) built with the oracle's
// restatement of the reference's scene pipeline, plus the reference's GPU packing
// (src/gpu.rs:37-119, :232-289, :346-381) so the tests can compare packed arrays.
//
// The draw protocol (SplitMix64, order of draws, defaults) is a project definition: the
// reference has no such scenes. The product's own scene builder follows the same protocol, and
// the tests check the two builders agree bit for bit.
#pragma once
#include <cstring>
#include <map>

#include "oracle_render.hpp"

namespace orc {

// SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number generators", 2014).
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double u01() { return (double)(next() >> 11) * 0x1.0p-53; }
    double uni(double a, double b) { return a + (b - a) * u01(); }
    // Uniform in the unit ball by rejection.
    void ball(double* v) {
        do {
            v[0] = uni(-1, 1); v[1] = uni(-1, 1); v[2] = uni(-1, 1);
        } while (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] >= 1.0);
    }
    double normal() {  // Box-Muller
        double u1 = 1.0 - u01(), u2 = u01();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// Mesh3D::uv_sphere's conventions (mesh4d.rs:508-563) applied to a subdivided icosahedron
// (the reference has no icosphere): unit directions from the 12 icosahedron vertices, each
// triangle split in 4 per level with normalized edge midpoints (first-created order), per
// triangle normal = normalized centroid, UV = (4 * longitude / 2pi, 2 * colatitude / pi) with the
// seam unwrapped per triangle.
struct IcoMesh {
    std::vector<std::array<double, 3>> v;
    std::vector<std::array<uint32_t, 3>> f;
};
inline IcoMesh icosphere_unit(int subdiv) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    IcoMesh m;
    const double raw[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                               {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : raw) {
        double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        m.v.push_back({p[0] / l, p[1] / l, p[2] / l});
    }
    m.f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
           {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int lvl = 0; lvl < subdiv; ++lvl) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
        auto midpoint = [&](uint32_t a, uint32_t b) -> uint32_t {
            auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            double x = m.v[a][0] + m.v[b][0], y = m.v[a][1] + m.v[b][1], z = m.v[a][2] + m.v[b][2];
            double l = std::sqrt(x * x + y * y + z * z);
            m.v.push_back({x / l, y / l, z / l});
            uint32_t idx = (uint32_t)m.v.size() - 1;
            mid[key] = idx;
            return idx;
        };
        std::vector<std::array<uint32_t, 3>> nf;
        for (auto& fc : m.f) {
            uint32_t a = fc[0], b = fc[1], c = fc[2];
            uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            nf.push_back({a, ab, ca});
            nf.push_back({b, bc, ab});
            nf.push_back({c, ca, bc});
            nf.push_back({ab, bc, ca});
        }
        m.f = nf;
    }
    return m;
}
template <class T> Mesh3D<T> icosphere(double radius, int subdiv) {
    IcoMesh im = icosphere_unit(subdiv);
    Mesh3D<T> out;
    for (auto& p : im.v) out.vertices.push_back(V3<T>((T)(radius * p[0]), (T)(radius * p[1]), (T)(radius * p[2])));
    const double PI = 3.141592653589793;
    for (auto& fc : im.f) {
        double us[3], vs[3];
        for (int k = 0; k < 3; ++k) {
            const auto& p = im.v[fc[k]];
            us[k] = 4.0 * (std::atan2(p[2], p[0]) / (2.0 * PI) + 0.5);
            vs[k] = 2.0 * std::acos(std::min(1.0, std::max(-1.0, p[1]))) / PI;
        }
        double umax = std::max(us[0], std::max(us[1], us[2])), umin = std::min(us[0], std::min(us[1], us[2]));
        if (umax - umin > 2.0)
            for (int k = 0; k < 3; ++k) if (us[k] < 2.0) us[k] += 4.0;
        Triangle3D<T> tri;
        tri.indices = fc;
        for (int k = 0; k < 3; ++k) tri.uv[k] = {(T)us[k], (T)vs[k]};
        V3<T> c = out.vertices[fc[0]] + out.vertices[fc[1]] + out.vertices[fc[2]];
        tri.normal = c.normalized();
        out.triangles.push_back(tri);
    }
    return out;
}

// Scene4D::common_materials (scene.rs:181-275).
template <class T> std::vector<Material<T>> common_materials() {
    auto mk = [](V3<T> b, V3<T> c, T em, T gs, T ww, Pattern p = CHECKERBOARD, T cav = T(1)) {
        Material<T> m;
        m.base_color = b; m.checker_color = c; m.emission = em; m.grid_scale = gs; m.wireframe_width = ww;
        m.pattern = p; m.cavity_length = cav;
        return m;
    };
    using V = V3<T>;
    std::vector<Material<T>> v;
    v.push_back(mk(V(T(0.22), T(0.25), T(0.30)), V(T(0.13), T(0.15), T(0.19)), T(0.18), T(1.0), T(0.012)));
    v.push_back(mk(V(T(0.20), T(0.72), T(0.95)), V(T(0.10), T(0.25), T(0.45)), T(0.28), T(1.0), T(0.025), CLOCK_FACE));
    v.push_back(mk(V(T(0.96), T(0.32), T(0.24)), V(T(0.45), T(0.12), T(0.10)), T(0.28), T(1.0), T(0.025), CLOCK_FACE));
    v.push_back(mk(V(T(0.96), T(0.78), T(0.20)), V(T(0.45), T(0.30), T(0.08)), T(0.28), T(1.0), T(0.025), CLOCK_FACE));
    v.push_back(mk(V(T(0.88), T(0.32), T(0.88)), V(T(0.32), T(0.10), T(0.38)), T(0.28), T(1.0), T(0.025), CLOCK_FACE));
    v.push_back(mk(V(T(0.20), T(0.95), T(0.65)), V(T(0.08), T(0.22), T(0.18)), T(0.32), T(1.0), T(0.025), LIGHT_CLOCK, T(1.0)));
    v.push_back(mk(V(T(0.85), T(0.82), T(0.72)), V(T(0.22), T(0.52), T(0.62)), T(0.18), T(2.0), T(0.025)));
    v.push_back(mk(V(T(0.25), T(0.92), T(1.00)), V(T(0.85), T(0.94), T(0.98)), T(0.28), T(2.0), T(0.030)));
    v.push_back(mk(V(T(0.96), T(0.38), T(0.22)), V(T(0.95), T(0.86), T(0.72)), T(0.22), T(2.0), T(0.030)));
    v.push_back(mk(V(T(1.00), T(0.10), T(0.025)), V(T(1.00), T(0.10), T(0.025)), T(1.20), T(1.0), T(0.0)));
    const T hull[4][3] = {{T(0.20), T(0.72), T(0.95)}, {T(0.96), T(0.32), T(0.24)}, {T(0.96), T(0.78), T(0.20)}, {T(0.88), T(0.32), T(0.88)}};
    for (auto& h : hull) v.push_back(mk(V(h[0], h[1], h[2]), V(h[0], h[1], h[2]), T(0.35), T(1.0), T(0.0)));
    return v;
}

// Parameters of a synthetic workload (mirrors SrSynthParams in include/specrel_scene.h).
struct SynthParams {
    uint32_t config = 1;   // 1 cubes, 2 icospheres, 3 translated cubes, 4 cubes (batch), 5 cubes + stars
    uint64_t seed = 1;
    uint32_t n_bodies = 64;
    uint32_t steps = 64;
    uint32_t subdiv = 2;
    uint32_t n_stars = 0;
    double translate[4] = {0, 0, 0, 0};
};

// Hyperbolic motion from rest at `t_acc` with proper acceleration `a` along `dir` for proper
// time `tau_acc`, then inertial (configuration 2's worldlines). Closed forms without
// cancellation: x(s) = a s^2 / (sqrt(1 + (a s)^2) + 1), v(s) = a s / sqrt(1 + (a s)^2).
struct HyperbolicPath {
    double c[3], dir[3], a, t_acc, t1, x1, v1;
    HyperbolicPath(const double* c_, const double* d_, double a_, double t_acc_, double tau_acc) {
        for (int i = 0; i < 3; ++i) { c[i] = c_[i]; dir[i] = d_[i]; }
        a = a_;
        t_acc = t_acc_;
        t1 = a > 1e-12 ? std::sinh(a * tau_acc) / a : 0.0;
        x1 = disp(t1);
        v1 = a > 1e-12 ? a * t1 / std::sqrt(1.0 + (a * t1) * (a * t1)) : 0.0;
    }
    double disp(double s) const { return a * s * s / (std::sqrt(1.0 + (a * s) * (a * s)) + 1.0); }
    Pos3d operator()(double t) const {
        double s = t - t_acc, x;
        if (s <= 0.0 || a <= 1e-12) x = 0.0;
        else if (s <= t1) x = disp(s);
        else x = x1 + v1 * (s - t1);
        return {c[0] + dir[0] * x, c[1] + dir[1] * x, c[2] + dir[2] * x};
    }
};

constexpr double ACCEL_START_T = -30.0;  // lab time the configuration-2 bodies start accelerating
constexpr double ACCEL_PROPER_TIME = 10.0;
constexpr double RINDLER_MARGIN = 0.8;   // |a| <= 0.8 / r keeps 1 + a.p > 0 with margin
constexpr double OBSERVER_CLEARANCE = 1.0;
constexpr double CUBE_RADIUS = 0.8660254037844386;  // half-diagonal of the unit cube

// Whether a body centre following `pos` stays farther than `dist` from the spatial origin (where
// the default observer stands) at the 51 lab times t = -5, -4.9, ..., 0.
template <class F> bool clear_of_observer(const F& pos, double dist) {
    for (int k = 0; k <= 50; ++k) {
        Pos3d q = pos(-5.0 + 0.1 * k);
        if (q.x * q.x + q.y * q.y + q.z * q.z < dist * dist) return false;
    }
    return true;
}

template <class T> struct SynthOut {
    Scene<T> scene;
    bool rindler_ok = true, superluminal = false;
    uint32_t clamped_accel = 0;  // bodies whose |a| was clamped for the Rindler horizon
    double cam_pos[4] = {0, 0, 0, 0};
    double cam_rapidity[3] = {0, 0, 0};
};

template <class T> SynthOut<T> synth_scene(const SynthParams& p) {
    SynthOut<T> out;
    SplitMix64 rng(p.seed);
    std::vector<Simplex<T>> simplices;
    auto& sc = out.scene;
    sc.materials = common_materials<T>();
    sc.light_pos = V3<T>(T(0), T(50), T(0));
    if (p.config == 2) {
        const uint32_t mats[6] = {6, 7, 8, 1, 6, 5};
        // The bodies are drawn in order (the draws alone use the generator), then extruded on
        // worker threads and concatenated in body order: the same simplices as one serial loop.
        struct Body { double c[3], d[3], r, a_eff; };
        std::vector<Body> bodies(p.n_bodies);
        for (uint32_t i = 0; i < p.n_bodies; ++i) {
            double c[3], r, a, d[3], a_eff;
            // A body that would enclose or graze the observer at the origin during t in [-5, 0]
            // is drawn again.
            for (int attempt = 0;; ++attempt) {
                c[0] = rng.uni(-20, 20); c[1] = rng.uni(-20, 20); c[2] = rng.uni(-20, 20);
                r = rng.uni(1, 3);
                a = rng.uni(0, 0.5);
                double dl2;
                do {
                    d[0] = rng.uni(-1, 1); d[1] = rng.uni(-1, 1); d[2] = rng.uni(-1, 1);
                    dl2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                } while (dl2 >= 1.0 || dl2 < 1e-6);
                double dl = std::sqrt(dl2);
                for (double& x : d) x /= dl;
                a_eff = std::min(a, RINDLER_MARGIN / r);
                HyperbolicPath probe(c, d, a_eff, ACCEL_START_T, ACCEL_PROPER_TIME);
                if (attempt >= 1000 || clear_of_observer(probe, r + OBSERVER_CLEARANCE)) break;
            }
            if (a_eff < a) out.clamped_accel++;
            Body& b = bodies[i];
            for (int k = 0; k < 3; ++k) { b.c[k] = c[k]; b.d[k] = d[k]; }
            b.r = r;
            b.a_eff = a_eff;
        }
        std::vector<std::vector<Simplex<T>>> parts(p.n_bodies);
        std::vector<char> sl(p.n_bodies, 0), ok(p.n_bodies, 1);
        parallel_for(p.n_bodies, [&](uint32_t i) {
            Body& b = bodies[i];
            HyperbolicPath path(b.c, b.d, b.a_eff, ACCEL_START_T, ACCEL_PROPER_TIME);
            bool s_l = false;
            auto samples = sample_accelerated_worldline<T>(path, T(-100), T(0), p.steps, &s_l);
            sl[i] = s_l;
            Mesh3D<T> mesh = icosphere<T>(b.r, (int)p.subdiv);
            ok[i] = extend_worldtube_simplices<T>(parts[i], mesh, samples, (const T*)nullptr, mats[i % 6]);
        });
        size_t total = 0;
        for (auto& v : parts) total += v.size();
        simplices.reserve(total);
        for (uint32_t i = 0; i < p.n_bodies; ++i) {
            out.superluminal |= sl[i] != 0;
            out.rindler_ok &= ok[i] != 0;
            simplices.insert(simplices.end(), parts[i].begin(), parts[i].end());
            std::vector<Simplex<T>>().swap(parts[i]);
        }
        double ph[3];
        rng.ball(ph);
        for (int k = 0; k < 3; ++k) out.cam_rapidity[k] = 2.0 * ph[k];
    } else {
        // Configurations 1, 3, 4 and 5 share the cube scene (64 inertial unit cubes).
        const uint32_t mats[3] = {6, 1, 5};
        Mesh3D<T> cube = Mesh3D<T>::cube(V3<T>(T(0.5), T(0.5), T(0.5)));
        for (uint32_t i = 0; i < p.n_bodies; ++i) {
            double c[3], b[3];
            for (int attempt = 0;; ++attempt) {
                c[0] = rng.uni(-20, 20); c[1] = rng.uni(-20, 20); c[2] = rng.uni(-20, 20);
                rng.ball(b);
                double cc[3] = {c[0], c[1], c[2]}, vv[3] = {0.9 * b[0], 0.9 * b[1], 0.9 * b[2]};
                auto line = [&](double t) { return Pos3d{cc[0] + vv[0] * t, cc[1] + vv[1] * t, cc[2] + vv[2] * t}; };
                if (attempt >= 1000 || clear_of_observer(line, CUBE_RADIUS + OBSERVER_CLEARANCE)) break;
            }
            V3<T> beta((T)(0.9 * b[0]), (T)(0.9 * b[1]), (T)(0.9 * b[2]));
            auto samples = sample_inertial_worldline<T>(V3<T>((T)c[0], (T)c[1], (T)c[2]), beta, T(-100), T(0), p.steps);
            if (p.translate[0] != 0 || p.translate[1] != 0 || p.translate[2] != 0 || p.translate[3] != 0)
                for (auto& s : samples)
                    s.center = s.center + V4<T>((T)p.translate[0], (T)p.translate[1], (T)p.translate[2], (T)p.translate[3]);
            out.rindler_ok &= extend_worldtube_simplices<T>(simplices, cube, samples, (const T*)nullptr, mats[i % 3]);
        }
        for (int k = 0; k < 4; ++k) out.cam_pos[k] = p.translate[k];
        // The translated scene carries its light with it.
        sc.light_pos = V3<T>((T)(0.0 + p.translate[1]), (T)(50.0 + p.translate[2]), (T)(0.0 + p.translate[3]));
        if (p.config == 5) {
            SplitMix64 srng(p.seed ^ 0x5354415253ull);
            for (uint32_t i = 0; i < p.n_stars; ++i) {
                double z = srng.uni(-1, 1), ph = srng.uni(0, 6.283185307179586);
                double rho = std::sqrt(std::max(0.0, 1.0 - z * z));
                double dir[3] = {rho * std::cos(ph), rho * std::sin(ph), z};
                double b[3];
                srng.ball(b);
                double temp = std::exp(srng.uni(std::log(2000.0), std::log(40000.0)));
                double inten = 1000.0 * 1000.0 * 2e-4 * std::exp(srng.normal());
                sc.stars.push_back(PointStar<T>::moving(
                    V3<T>((T)(1000.0 * dir[0]), (T)(1000.0 * dir[1]), (T)(1000.0 * dir[2])),
                    V3<T>((T)(0.01 * b[0]), (T)(0.01 * b[1]), (T)(0.01 * b[2])), (T)temp, (T)inten));
            }
            out.cam_rapidity[0] = 0.8;
            out.cam_rapidity[1] = -0.3;
            out.cam_rapidity[2] = 0.5;
        }
    }
    sc.bvh = Bvh<T>::build(std::move(simplices));
    sc.finish_stars();
    return out;
}

// One observer of the batched workload (configuration 4).
struct ObserverDraw {
    uint32_t width, height;
    double pos[4];
    double rapidity[3];
    uint32_t slice_mode;  // 0 past light cone, 1 God's-eye slice
};
inline std::vector<ObserverDraw> synth_observers(uint64_t seed, uint32_t n) {
    SplitMix64 rng(seed ^ 0x4F4253ull);
    const uint32_t RES[4][2] = {{320, 200}, {640, 400}, {1280, 800}, {1920, 1200}};
    std::vector<ObserverDraw> out;
    for (uint32_t i = 0; i < n; ++i) {
        ObserverDraw o;
        uint32_t ri = std::min<uint32_t>(3, (uint32_t)(rng.u01() * 4.0));
        o.width = RES[ri][0];
        o.height = RES[ri][1];
        o.pos[0] = rng.uni(-50, 0);
        double x[3];
        rng.ball(x);
        for (int k = 0; k < 3; ++k) o.pos[1 + k] = 30.0 * x[k];
        rng.ball(x);
        for (int k = 0; k < 3; ++k) o.rapidity[k] = 3.0 * x[k];
        o.slice_mode = rng.u01() < 0.5 ? 0u : 1u;
        out.push_back(o);
    }
    return out;
}

// ------------------------------------------------------------------------------------------
// The reference's GPU packing (gpu.rs:44-119, :247-289, :346-381), float scenes only.
// ------------------------------------------------------------------------------------------
struct PNode { float min[4], max[4]; uint32_t right_or_first, count, left, pad; };
struct PGeom { float v0[4], n[4], b1[4], b2[4], b3[4]; };
struct PAttr { float uv_u[4], uv_v[4], tb_x[4], tb_y[4], tb_z[4], tau[4], grad_u[4], grad_v[4], normal[4], four_vel[4], misc[4], decided_at[4]; };
struct PMat { float base[4], checker[4], params[4]; };
static_assert(sizeof(PNode) == 48 && sizeof(PGeom) == 80 && sizeof(PAttr) == 192 && sizeof(PMat) == 48, "layout");

inline void v4f(float* d, const V4<float>& v) { d[0] = v.t; d[1] = v.x; d[2] = v.y; d[3] = v.z; }
inline float bits_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

inline void pack_scene(const Scene<float>& s, PNode* nodes, PGeom* geoms, PAttr* attrs, PMat* mats, float* stars,
                       uint32_t* order) {
    const auto& b = s.bvh;
    for (size_t i = 0; i < b.nodes.size(); ++i) {
        PNode& n = nodes[i];
        v4f(n.min, b.nodes[i].aabb.min);
        v4f(n.max, b.nodes[i].aabb.max);
        n.right_or_first = b.nodes[i].right_or_first;
        n.count = b.nodes[i].count;
        n.left = b.nodes[i].left;
        n.pad = 0;
    }
    for (size_t i = 0; i < b.hot.size(); ++i) {
        const auto& g = b.hot[i];
        v4f(geoms[i].v0, g.v0); v4f(geoms[i].n, g.n); v4f(geoms[i].b1, g.b1); v4f(geoms[i].b2, g.b2); v4f(geoms[i].b3, g.b3);
        const auto& sx = b.leaf_simplex(i);
        PAttr& a = attrs[i];
        for (int k = 0; k < 4; ++k) {
            a.uv_u[k] = sx.uv_u[k]; a.uv_v[k] = sx.uv_v[k];
            a.tb_x[k] = sx.tri_bary[k].x; a.tb_y[k] = sx.tri_bary[k].y; a.tb_z[k] = sx.tri_bary[k].z;
            a.tau[k] = sx.tau[k]; a.grad_u[k] = sx.grad_u[k]; a.grad_v[k] = sx.grad_v[k];
            a.decided_at[k] = sx.decided_at[k];
        }
        v4f(a.normal, sx.normal);
        v4f(a.four_vel, sx.four_vel);
        a.misc[0] = sx.uvs_u; a.misc[1] = sx.uvs_v; a.misc[2] = bits_f(sx.material_id); a.misc[3] = 0;
        if (order) order[i] = b.order[i];
    }
    for (size_t i = 0; i < s.materials.size(); ++i) {
        const auto& m = s.materials[i];
        PMat& pm = mats[i];
        pm.base[0] = m.base_color.x; pm.base[1] = m.base_color.y; pm.base[2] = m.base_color.z; pm.base[3] = m.emission;
        pm.checker[0] = m.checker_color.x; pm.checker[1] = m.checker_color.y; pm.checker[2] = m.checker_color.z; pm.checker[3] = m.grid_scale;
        pm.params[0] = m.wireframe_width; pm.params[1] = bits_f((uint32_t)m.pattern); pm.params[2] = m.cavity_length; pm.params[3] = 0;
    }
    if (stars) {  // gpu.rs:106-119
        size_t w = 0;
        uint32_t first = 0;
        for (size_t i = 0; i < s.stars.size(); ++i) {
            uint32_t cnt = (uint32_t)s.stars[i].segments.size();
            stars[w++] = s.stars[i].temperature; stars[w++] = s.star_cn[i]; stars[w++] = bits_f(first); stars[w++] = bits_f(cnt);
            first += cnt;
        }
        for (auto& st : s.stars)
            for (auto& seg : st.segments) {
                v4f(&stars[w], seg.event); w += 4;
                v4f(&stars[w], seg.four_velocity); w += 4;
                stars[w++] = seg.s_min; stars[w++] = seg.s_max; stars[w++] = 0; stars[w++] = 0;
            }
    }
}

}  // namespace orc
