// Caller-side scene pipeline for the seeded synthetic workloads: meshes, worldlines, worldtube
// extrusion into 4D tetrahedra, the 8-bin 4-axis SAH BVH, and the reference's GPU packing.
//
// Restates, for f32 scenes:
//   mesh4d.rs:312-371  Simplex4D::new          mesh4d.rs:453-505  Mesh3D::cube
//   mesh4d.rs:663-854  worldtube extrusion     mesh4d.rs:912-1052 inertial / accelerated worldlines
//   bvh4d.rs:8-13, 123-141, 254-427  box_measure, build, build_subtree, split
//   gpu.rs:106-119, 247-289, 346-381 pack_stars, PackedSceneGpuData::from_scene, GpuAttr::pack
//   star.rs:85-124 PointStar::moving, color_norm; scene.rs:181-275 common_materials
// Worldtubes of different bodies are extruded on worker threads and concatenated in body order,
// and BVH subtrees of at least 4096 primitives are built concurrently and spliced depth-first,
// so the arrays are identical to a serial build's.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/specrel_scene.h"
#include "sr_math.hpp"
#include "rust_select.hpp"
#include "tube_build.hpp"

using namespace srh;

namespace {

struct Rng {  // SplitMix64 (Steele, Lea & Flood 2014)
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double u01() { return (double)(next() >> 11) * 0x1.0p-53; }
    double uni(double a, double b) { return a + (b - a) * u01(); }
    void ball(double* v) {
        do { v[0] = uni(-1, 1); v[1] = uni(-1, 1); v[2] = uni(-1, 1); } while (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] >= 1.0);
    }
    double normal() {
        double u1 = 1.0 - u01(), u2 = u01();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct Tri { uint32_t idx[3]; float uv[3][2]; V3f normal; };
struct Mesh { std::vector<V3f> v; std::vector<Tri> tris; };

Mesh cube_mesh(float he) {  // mesh4d.rs:454-505 with equal half-extents
    Mesh m;
    for (float z : {-he, he}) for (float y : {-he, he}) for (float x : {-he, he}) m.v.push_back(V3f(x, y, z));
    const float us = std::fmax(std::round(he / std::fmax(he, 1e-4f)), 1.0f);
    const uint32_t F[6][4] = {{0, 1, 3, 2}, {5, 4, 6, 7}, {4, 0, 2, 6}, {1, 5, 7, 3}, {4, 5, 1, 0}, {2, 3, 7, 6}};
    const V3f N[6] = {V3f(0, 0, -1), V3f(0, 0, 1), V3f(-1, 0, 0), V3f(1, 0, 0), V3f(0, -1, 0), V3f(0, 1, 0)};
    for (int f = 0; f < 6; ++f) {
        const float q[4][2] = {{0, 0}, {us, 0}, {us, 1}, {0, 1}};
        Tri a{{F[f][0], F[f][1], F[f][2]}, {{q[0][0], q[0][1]}, {q[1][0], q[1][1]}, {q[2][0], q[2][1]}}, N[f]};
        Tri b{{F[f][0], F[f][2], F[f][3]}, {{q[0][0], q[0][1]}, {q[2][0], q[2][1]}, {q[3][0], q[3][1]}}, N[f]};
        m.tris.push_back(a);
        m.tris.push_back(b);
    }
    return m;
}

// Icosahedron subdivided `subdiv` times; uv_sphere's UV convention (mesh4d.rs:508-563).
Mesh icosphere_mesh(double radius, int subdiv) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<std::array<double, 3>> v;
    const double raw[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                               {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : raw) {
        double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        v.push_back({p[0] / l, p[1] / l, p[2] / l});
    }
    std::vector<std::array<uint32_t, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                                              {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                                              {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int lvl = 0; lvl < subdiv; ++lvl) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> cache;
        auto mid = [&](uint32_t a, uint32_t b) {
            auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = cache.find(key);
            if (it != cache.end()) return it->second;
            double x = v[a][0] + v[b][0], y = v[a][1] + v[b][1], z = v[a][2] + v[b][2];
            double l = std::sqrt(x * x + y * y + z * z);
            v.push_back({x / l, y / l, z / l});
            return cache[key] = (uint32_t)v.size() - 1;
        };
        std::vector<std::array<uint32_t, 3>> nf;
        nf.reserve(f.size() * 4);
        for (auto& c : f) {
            uint32_t ab = mid(c[0], c[1]), bc = mid(c[1], c[2]), ca = mid(c[2], c[0]);
            nf.push_back({c[0], ab, ca});
            nf.push_back({c[1], bc, ab});
            nf.push_back({c[2], ca, bc});
            nf.push_back({ab, bc, ca});
        }
        f.swap(nf);
    }
    Mesh m;
    for (auto& p : v) m.v.push_back(V3f((float)(radius * p[0]), (float)(radius * p[1]), (float)(radius * p[2])));
    const double PI = 3.141592653589793;
    for (auto& c : f) {
        Tri tr;
        double us[3], vs[3];
        for (int k = 0; k < 3; ++k) {
            tr.idx[k] = c[k];
            const auto& p = v[c[k]];
            us[k] = 4.0 * (std::atan2(p[2], p[0]) / (2.0 * PI) + 0.5);
            vs[k] = 2.0 * std::acos(std::min(1.0, std::max(-1.0, p[1]))) / PI;
        }
        double hi = std::max(us[0], std::max(us[1], us[2])), lo = std::min(us[0], std::min(us[1], us[2]));
        if (hi - lo > 2.0)
            for (double& u : us) if (u < 2.0) u += 4.0;
        for (int k = 0; k < 3; ++k) { tr.uv[k][0] = (float)us[k]; tr.uv[k][1] = (float)vs[k]; }
        tr.normal = (m.v[c[0]] + m.v[c[1]] + m.v[c[2]]).normalized();
        m.tris.push_back(tr);
    }
    return m;
}

struct Sample { V4f center; float tau; V3f phi, accel; Tetrad<float> tet; };

std::vector<Sample> inertial_worldline(V3f pos, V3f beta, float t_min, float t_max, size_t steps) {  // mesh4d.rs:912-937
    Tetrad<float> tet = Tetrad<float>::from_beta(beta);
    double inv_gamma = 1.0 / (double)tet.e[0].t;
    std::vector<Sample> out;
    for (size_t i = 0; i <= steps; ++i) {
        double t = (double)t_min + ((double)i / (double)steps) * (double)(t_max - t_min);
        V3f p = pos + beta * (float)t;
        out.push_back({V4f((float)t, p.x, p.y, p.z), (float)(t * inv_gamma), V3f(), V3f(), tet});
    }
    return out;
}

struct P3 { double x, y, z; };
// mesh4d.rs:947-1052.
std::vector<Sample> accelerated_worldline(const std::function<P3(double)>& pos, float t_min, float t_max, size_t steps) {
    const double h = 1e-5;
    auto vel = [&](double t) {
        P3 a = pos(t - h), b = pos(t + h);
        double k = 0.5 / h;
        return P3{(b.x - a.x) * k, (b.y - a.y) * k, (b.z - a.z) * k};
    };
    auto fourvel = [&](double t, V4f* u) {
        P3 v = vel(t);
        double b2 = std::min(v.x * v.x + v.y * v.y + v.z * v.z, 0.999999999);
        double ig = std::sqrt(1.0 - b2), g = 1.0 / ig;
        *u = V4f((float)g, (float)(g * v.x), (float)(g * v.y), (float)(g * v.z));
        return ig;
    };
    auto accel_world = [&](double t) {
        V4f u0, um, up;
        double ig = fourvel(t, &u0);
        fourvel(t - h, &um);
        fourvel(t + h, &up);
        return ((up - um) * (0.5f / (float)h)) * (1.0f / (float)ig);
    };
    double t0 = (double)t_min, span = (double)(t_max - t_min);
    P3 v0 = vel(t0);
    Tetrad<float> tet = Tetrad<float>::from_beta(V3f((float)v0.x, (float)v0.y, (float)v0.z));
    double tau = 0.0, prev = t0;
    V3f phi;
    std::vector<Sample> out;
    for (size_t i = 0; i <= steps; ++i) {
        double t = t0 + ((double)i / (double)steps) * span;
        if (i > 0) {
            double sub = (t - prev) / 8.0;
            for (int s = 0; s < 8; ++s) {
                double ta = prev + (double)s * sub, tb = ta + sub, tm = 0.5 * (ta + tb);
                V4f ua, um, ub;
                double ia = fourvel(ta, &ua), im = fourvel(tm, &um), ib = fourvel(tb, &ub);
                tau += (sub / 6.0) * (ia + 4.0 * im + ib);
                V4f du = ub - ua;
                V3f before = tet.world_to_local_spatial(du);
                tet.boost_to(ub);
                V3f after = tet.world_to_local_spatial(du);
                phi += (before + after) * 0.5f;
            }
        }
        prev = t;
        P3 p = pos(t);
        out.push_back({V4f((float)t, (float)p.x, (float)p.y, (float)p.z), (float)tau, phi,
                       tet.world_to_local_spatial(accel_world(t)), tet});
    }
    return out;
}

// extend_worldtube_simplices (mesh4d.rs:721-854), static geometry (decided_at = -1e9): the
// worldtube's events at every sample, then the three tetrahedra of each triangle between
// consecutive samples (tube_segment, shared with the device build).
TubeSample tube_sample(const Sample& smp) {
    TubeSample t;
    t.center = smp.center;
    t.tau = smp.tau;
    t.phi = smp.phi;
    t.accel = smp.accel;
    for (int k = 0; k < 4; ++k) t.e[k] = smp.tet.e[k];
    return t;
}

bool extrude(std::vector<Tet>& out, const Mesh& mesh, const std::vector<Sample>& s, uint32_t mat) {
    size_t nv = mesh.v.size();
    bool rindler_ok = true;
    std::vector<TubeSample> ts;
    for (auto& smp : s) ts.push_back(tube_sample(smp));
    std::vector<V4f> ev;
    ev.reserve(s.size() * nv);
    for (auto& smp : ts)
        for (auto& p : mesh.v) {
            if (!(1.0f + smp.accel.dot(p) > 0.0f)) rindler_ok = false;
            ev.push_back(smp.center + to_world(smp, p));
        }
    std::vector<TubeTri> tt;
    for (auto& tr : mesh.tris) tt.push_back(make_tube_tri(mesh.v.data(), tr.idx, tr.uv, tr.normal));
    out.reserve(out.size() + (s.size() - 1) * 3 * tt.size());
    for (size_t st = 0; st + 1 < s.size(); ++st)
        for (auto& t : tt) {
            Tet tet[3];
            bool ok[3];
            tube_segment(t, &ev[st * nv], &ev[(st + 1) * nv], ts[st], ts[st + 1], mat, DECIDED_STATIC, DECIDED_STATIC, tet,
                         ok);
            for (int k = 0; k < 3; ++k)
                if (ok[k]) out.push_back(tet[k]);
        }
    return rindler_ok;
}

// ---------------------------------------------------------------------------------------------
// 4D SAH BVH (bvh4d.rs).
// ---------------------------------------------------------------------------------------------
struct Ref { Box box; V4f c; uint32_t index; };
struct Node { Box box; uint32_t right_or_first, count, left; };

inline float box_measure(const Box& b) {  // bvh4d.rs:8-13
    V4f e = b.hi - b.lo;
    return e.x * e.y + e.y * e.z + e.z * e.x + 0.22f * e.t * (e.x + e.y + e.z);
}

struct Builder {
    unsigned spawn_depth;  // subtrees above this recursion depth may build their halves concurrently
    std::atomic<uint32_t>* median = nullptr;  // counts the splits that fell back to the median

    static inline uint64_t sat_usize(float x) { return (std::isnan(x) || x <= 0.0f) ? 0 : (uint64_t)x; }

    struct Bins { Box box[4][8]; uint32_t cnt[4][8]; };

    // bvh4d.rs:307-427; returns false for a leaf. Folds over large nodes run on worker threads
    // (box unions and counts merge exactly, so the result does not depend on the chunking).
    bool split(Ref* r, size_t n, Box* bounds_out, size_t* mid_out, unsigned depth) const {
        auto fold_bounds = [&](size_t lo, size_t hi) {
            Box b, cb;
            for (size_t i = lo; i < hi; ++i) { b = unite(b, r[i].box); grow(cb, r[i].c); }
            return std::make_pair(b, cb);
        };
        const size_t CHUNK = 1 << 16;
        bool par = n >= 4 * CHUNK && depth < spawn_depth;
        Box bounds, cb;
        if (par) {
            size_t parts = (n + CHUNK - 1) / CHUNK;
            std::vector<std::future<std::pair<Box, Box>>> fs;
            for (size_t p = 0; p < parts; ++p)
                fs.push_back(std::async(std::launch::async, fold_bounds, p * CHUNK, std::min(n, (p + 1) * CHUNK)));
            for (auto& f : fs) { auto x = f.get(); bounds = unite(bounds, x.first); cb = unite(cb, x.second); }
        } else {
            auto x = fold_bounds(0, n);
            bounds = x.first;
            cb = x.second;
        }
        *bounds_out = bounds;
        if (n <= 3) return false;
        V4f ext = cb.hi - cb.lo;
        bool live[4];
        float amin[4], inv[4];
        for (int a = 0; a < 4; ++a) { live[a] = ext.ax(a) >= 1e-4f; amin[a] = cb.lo.ax(a); inv[a] = 8.0f / ext.ax(a); }
        auto fold_bins = [&](size_t lo, size_t hi) {
            Bins b{};
            for (size_t i = lo; i < hi; ++i)
                for (int a = 0; a < 4; ++a) {
                    if (!live[a]) continue;
                    uint64_t k = std::min<uint64_t>(sat_usize((r[i].c.ax(a) - amin[a]) * inv[a]), 7);
                    b.box[a][k] = unite(b.box[a][k], r[i].box);
                    b.cnt[a][k] += 1;
                }
            return b;
        };
        Bins bins{};
        if (par) {
            size_t parts = (n + CHUNK - 1) / CHUNK;
            std::vector<std::future<Bins>> fs;
            for (size_t p = 0; p < parts; ++p)
                fs.push_back(std::async(std::launch::async, fold_bins, p * CHUNK, std::min(n, (p + 1) * CHUNK)));
            for (auto& f : fs) {
                Bins x = f.get();
                for (int a = 0; a < 4; ++a)
                    for (int k = 0; k < 8; ++k) { bins.box[a][k] = unite(bins.box[a][k], x.box[a][k]); bins.cnt[a][k] += x.cnt[a][k]; }
            }
        } else {
            bins = fold_bins(0, n);
        }
        int best_axis = 0;
        float best_pos = 0, best_cost = INFINITY;
        for (int a = 0; a < 4; ++a) {
            if (!live[a]) continue;
            Box lb[7], cur;
            uint32_t lc[7], cc = 0;
            for (int i = 0; i < 7; ++i) { cur = unite(cur, bins.box[a][i]); cc += bins.cnt[a][i]; lb[i] = cur; lc[i] = cc; }
            Box rb;
            uint32_t rc = 0;
            for (int i = 6; i >= 0; --i) {
                rb = unite(rb, bins.box[a][i + 1]);
                rc += bins.cnt[a][i + 1];
                if (lc[i] > 0 && rc > 0) {
                    float cost = (float)lc[i] * box_measure(lb[i]) + (float)rc * box_measure(rb);
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = a;
                        best_pos = amin[a] + ((float)(i + 1) / 8.0f) * ext.ax(a);
                    }
                }
            }
        }
        if (best_cost == INFINITY) {
            float me = -1.0f;
            for (int a = 0; a < 4; ++a) if (ext.ax(a) > me) { me = ext.ax(a); best_axis = a; }
            if (me < 1e-5f) return false;
            best_pos = ((cb.lo + cb.hi) * 0.5f).ax(best_axis);
        }
        size_t mid = 0;
        for (size_t i = 0; i < n; ++i)
            if (r[i].c.ax(best_axis) < best_pos) { std::swap(r[i], r[mid]); ++mid; }
        if (mid == 0 || mid == n) {  // bvh4d.rs:418-424: select_nth_unstable_by on the centroid
            mid = n / 2;
            sr_select::select_nth_unstable(r, n, mid, [best_axis](const Ref& a, const Ref& b) {
                return a.c.ax(best_axis) < b.c.ax(best_axis);  // partial_cmp == Less (no NaN centroids)
            });
            if (median) median->fetch_add(1, std::memory_order_relaxed);
        }
        *mid_out = mid;
        return true;
    }

    // Serial build appending depth-first with absolute links (bvh4d.rs:287-303).
    uint32_t build_rec(std::vector<Node>& nodes, Ref* r, size_t n, size_t first) const {
        uint32_t idx = (uint32_t)nodes.size();
        Box b;
        size_t mid;
        if (!split(r, n, &b, &mid, UINT32_MAX)) {
            nodes.push_back({b, (uint32_t)first, (uint32_t)n, 0});
            return idx;
        }
        nodes.push_back({b, 0, 0, idx + 1});
        build_rec(nodes, r, mid, first);
        uint32_t right = build_rec(nodes, r + mid, n - mid, first + mid);
        nodes[idx].right_or_first = right;
        return idx;
    }

    // The subtree over r as its own array (root first, links relative to it); halves of large
    // subtrees build concurrently and are spliced back depth-first (bvh4d.rs:257-279).
    std::vector<Node> build_sub(Ref* r, size_t n, size_t first, unsigned depth) const {
        if (n < 4096 || depth >= spawn_depth) {
            std::vector<Node> nodes;
            nodes.reserve(n);
            build_rec(nodes, r, n, first);
            return nodes;
        }
        Box b;
        size_t mid;
        if (!split(r, n, &b, &mid, depth)) return {Node{b, (uint32_t)first, (uint32_t)n, 0}};
        auto fl = std::async(std::launch::async, [&] { return build_sub(r, mid, first, depth + 1); });
        std::vector<Node> right = build_sub(r + mid, n - mid, first + mid, depth + 1);
        std::vector<Node> left = fl.get();
        uint32_t ri = 1 + (uint32_t)left.size();
        std::vector<Node> out;
        out.reserve(1 + left.size() + right.size());
        out.push_back({b, ri, 0, 1});
        for (auto x : left) { if (x.count == 0) { x.left += 1; x.right_or_first += 1; } out.push_back(x); }
        for (auto x : right) { if (x.count == 0) { x.left += ri; x.right_or_first += ri; } out.push_back(x); }
        return out;
    }
};

}  // namespace

struct sr_scene {
    std::vector<SrGpuNode> nodes;
    std::vector<SrGpuGeom> geoms;
    std::vector<SrGpuAttr> attrs;
    std::vector<SrGpuMaterial> mats;
    std::vector<float> stars;
    std::vector<uint32_t> order;
    std::vector<float> boxes;  // build order: min (t, x, y, z), max (t, x, y, z) per simplex
    struct TubeRec {
        std::vector<float> verts;
        std::vector<SrTubeTriangle> tris;
        std::vector<SrTubeSample> samples;
        uint32_t mat = 0;
    };
    std::vector<TubeRec> tube_recs;  // the bodies' worldtubes (sr_scene_tubes)
    std::vector<SrTube> tubes;
    uint32_t num_stars = 0;
    double anchor[4] = {0, 0, 0, 0};
    SrSynthInfo info{};
};

static void set_err(char* err, size_t len, const std::string& m) {
    if (err && len) { std::strncpy(err, m.c_str(), len - 1); err[len - 1] = 0; }
}

static std::vector<SrGpuMaterial> common_materials() {  // scene.rs:181-275
    struct M { float b[3], c[3], em, gs, ww; uint32_t pat; float cav; };
    const M ms[14] = {
        {{0.22f, 0.25f, 0.30f}, {0.13f, 0.15f, 0.19f}, 0.18f, 1.0f, 0.012f, 0, 1.0f},
        {{0.20f, 0.72f, 0.95f}, {0.10f, 0.25f, 0.45f}, 0.28f, 1.0f, 0.025f, 1, 1.0f},
        {{0.96f, 0.32f, 0.24f}, {0.45f, 0.12f, 0.10f}, 0.28f, 1.0f, 0.025f, 1, 1.0f},
        {{0.96f, 0.78f, 0.20f}, {0.45f, 0.30f, 0.08f}, 0.28f, 1.0f, 0.025f, 1, 1.0f},
        {{0.88f, 0.32f, 0.88f}, {0.32f, 0.10f, 0.38f}, 0.28f, 1.0f, 0.025f, 1, 1.0f},
        {{0.20f, 0.95f, 0.65f}, {0.08f, 0.22f, 0.18f}, 0.32f, 1.0f, 0.025f, 2, 1.0f},
        {{0.85f, 0.82f, 0.72f}, {0.22f, 0.52f, 0.62f}, 0.18f, 2.0f, 0.025f, 0, 1.0f},
        {{0.25f, 0.92f, 1.00f}, {0.85f, 0.94f, 0.98f}, 0.28f, 2.0f, 0.030f, 0, 1.0f},
        {{0.96f, 0.38f, 0.22f}, {0.95f, 0.86f, 0.72f}, 0.22f, 2.0f, 0.030f, 0, 1.0f},
        {{1.00f, 0.10f, 0.025f}, {1.00f, 0.10f, 0.025f}, 1.20f, 1.0f, 0.0f, 0, 1.0f},
        {{0.20f, 0.72f, 0.95f}, {0.20f, 0.72f, 0.95f}, 0.35f, 1.0f, 0.0f, 0, 1.0f},
        {{0.96f, 0.32f, 0.24f}, {0.96f, 0.32f, 0.24f}, 0.35f, 1.0f, 0.0f, 0, 1.0f},
        {{0.96f, 0.78f, 0.20f}, {0.96f, 0.78f, 0.20f}, 0.35f, 1.0f, 0.0f, 0, 1.0f},
        {{0.88f, 0.32f, 0.88f}, {0.88f, 0.32f, 0.88f}, 0.35f, 1.0f, 0.0f, 0, 1.0f},
    };
    std::vector<SrGpuMaterial> out;
    for (auto& m : ms) {
        SrGpuMaterial g{};
        for (int k = 0; k < 3; ++k) { g.base[k] = m.b[k]; g.checker[k] = m.c[k]; }
        g.base[3] = m.em;
        g.checker[3] = m.gs;
        g.params[0] = m.ww;
        g.params[1] = fbits(m.pat);
        g.params[2] = m.cav;
        out.push_back(g);
    }
    return out;
}

// Blackbody colour normalisation of a star (star.rs:117-124, 156-180); the powi(5) of the
// constant primary wavelengths is folded once in double precision, as the compiled reference does.
static float planck(float lam, float temp) {
    float x = std::fmin(14388.0f / (lam * std::fmax(temp, 1.0f)), 80.0f);
    return 1.0f / ((float)std::pow((double)lam, 5.0) * (std::exp(x) - 1.0f));
}
static float color_norm(float temp, float inten) {
    const float W = 6504.0f;
    float r = planck(0.610f, temp) / planck(0.610f, W), g = planck(0.550f, temp) / planck(0.550f, W),
          b = planck(0.465f, temp) / planck(0.465f, W);
    float lum = 0.2126f * r + 0.7152f * g + 0.0722f * b;
    return lum > 0.0f ? inten / lum : 0.0f;
}

extern "C" sr_status sr_scene_synth(const SrSynthParams* p, sr_scene** out, char* err, size_t errlen) {
    if (!p || !out) { set_err(err, errlen, "null argument"); return SR_ERR_INVALID_ARGUMENT; }
    if (p->config < 1 || p->config > 5 || p->n_bodies == 0 || p->steps == 0) {
        set_err(err, errlen, "config must be 1..5 with n_bodies > 0 and steps > 0");
        return SR_ERR_INVALID_ARGUMENT;
    }
    auto t_start = std::chrono::steady_clock::now();
    unsigned threads = p->threads ? p->threads : std::max(1u, std::thread::hardware_concurrency());
    auto sc = std::make_unique<sr_scene>();
    Rng rng{p->seed};
    std::vector<std::vector<Tet>> per_body(p->n_bodies);
    using TubeRec = sr_scene::TubeRec;
    // A body's worldtube as recorded for sr_scene_tubes.
    auto record = [](TubeRec& rec, const Mesh& m, const std::vector<Sample>& smp, uint32_t mat) {
        for (auto& v : m.v) { rec.verts.push_back(v.x); rec.verts.push_back(v.y); rec.verts.push_back(v.z); }
        for (auto& t : m.tris) {
            SrTubeTriangle x{};
            for (int k = 0; k < 3; ++k) { x.idx[k] = t.idx[k]; x.uv[k][0] = t.uv[k][0]; x.uv[k][1] = t.uv[k][1]; }
            x.normal[0] = t.normal.x; x.normal[1] = t.normal.y; x.normal[2] = t.normal.z;
            rec.tris.push_back(x);
        }
        for (auto& q : smp) {
            SrTubeSample x{};
            put4(x.center, q.center);
            for (int k = 0; k < 4; ++k) put4(x.tetrad[k], q.tet.e[k]);
            x.proper_time = q.tau;
            x.phi[0] = q.phi.x; x.phi[1] = q.phi.y; x.phi[2] = q.phi.z;
            x.accel[0] = q.accel.x; x.accel[1] = q.accel.y; x.accel[2] = q.accel.z;
            rec.samples.push_back(x);
        }
        rec.mat = mat;
    };
    std::vector<std::function<bool(std::vector<Tet>&, TubeRec&)>> jobs;
    // A body that would enclose or graze the observer standing at the spatial origin (within its
    // radius + 1 of it at the lab times -5, -4.9, ..., 0) is drawn again.
    auto clear_of_observer = [](const std::function<P3(double)>& pos, double dist) {
        for (int k = 0; k <= 50; ++k) {
            P3 q = pos(-5.0 + 0.1 * k);
            if (q.x * q.x + q.y * q.y + q.z * q.z < dist * dist) return false;
        }
        return true;
    };
    if (p->config == 2) {
        const uint32_t mats[6] = {6, 7, 8, 1, 6, 5};
        for (uint32_t i = 0; i < p->n_bodies; ++i) {
            double c[3], r, a, d[3], ae, t1, x1, v1;
            // Hyperbolic motion from rest at t = -30 for proper time 10, then inertial, with
            // |a| clamped to 0.8 / r so every vertex stays inside its Rindler horizon.
            auto disp = [](double ae_, double s) { return ae_ * s * s / (std::sqrt(1.0 + (ae_ * s) * (ae_ * s)) + 1.0); };
            auto path_of = [&](const double* cc, const double* dd) {
                std::array<double, 3> c3{cc[0], cc[1], cc[2]}, d3{dd[0], dd[1], dd[2]};
                double ae_ = ae, t1_ = t1, x1_ = x1, v1_ = v1;
                return std::function<P3(double)>([=](double t) {
                    double s = t - (-30.0), x;
                    if (s <= 0.0 || ae_ <= 1e-12) x = 0.0;
                    else if (s <= t1_) x = ae_ * s * s / (std::sqrt(1.0 + (ae_ * s) * (ae_ * s)) + 1.0);
                    else x = x1_ + v1_ * (s - t1_);
                    return P3{c3[0] + d3[0] * x, c3[1] + d3[1] * x, c3[2] + d3[2] * x};
                });
            };
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
                ae = std::min(a, 0.8 / r);
                t1 = ae > 1e-12 ? std::sinh(ae * 10.0) / ae : 0.0;
                x1 = disp(ae, t1);
                v1 = ae > 1e-12 ? ae * t1 / std::sqrt(1.0 + (ae * t1) * (ae * t1)) : 0.0;
                if (attempt >= 1000 || clear_of_observer(path_of(c, d), r + 1.0)) break;
            }
            if (ae < a) sc->info.clamped_accel++;
            auto pos = path_of(c, d);
            uint32_t mat = mats[i % 6], steps = p->steps, subdiv = p->subdiv;
            jobs.push_back([=](std::vector<Tet>& o, TubeRec& rec) {
                Mesh m = icosphere_mesh(r, (int)subdiv);
                std::vector<Sample> smp = accelerated_worldline(pos, -100.0f, 0.0f, steps);
                record(rec, m, smp, mat);
                return extrude(o, m, smp, mat);
            });
        }
        double ph[3];
        rng.ball(ph);
        for (int k = 0; k < 3; ++k) sc->info.cam_rapidity[k] = 2.0 * ph[k];
    } else {
        const uint32_t mats[3] = {6, 1, 5};
        for (uint32_t i = 0; i < p->n_bodies; ++i) {
            double c[3], b[3];
            for (int attempt = 0;; ++attempt) {
                c[0] = rng.uni(-20, 20); c[1] = rng.uni(-20, 20); c[2] = rng.uni(-20, 20);
                rng.ball(b);
                std::array<double, 3> cc{c[0], c[1], c[2]}, vv{0.9 * b[0], 0.9 * b[1], 0.9 * b[2]};
                std::function<P3(double)> line = [=](double t) {
                    return P3{cc[0] + vv[0] * t, cc[1] + vv[1] * t, cc[2] + vv[2] * t};
                };
                if (attempt >= 1000 || clear_of_observer(line, 0.8660254037844386 + 1.0)) break;
            }
            V3f pos((float)c[0], (float)c[1], (float)c[2]);
            V3f beta((float)(0.9 * b[0]), (float)(0.9 * b[1]), (float)(0.9 * b[2]));
            uint32_t mat = mats[i % 3], steps = p->steps;
            jobs.push_back([=](std::vector<Tet>& o, TubeRec& rec) {
                Mesh m = cube_mesh(0.5f);
                std::vector<Sample> smp = inertial_worldline(pos, beta, -100.0f, 0.0f, steps);
                record(rec, m, smp, mat);
                return extrude(o, m, smp, mat);
            });
        }
        // Configuration 3: the same f32 scene, whose coordinates are relative to the FP64 anchor.
        if (p->config == 3)
            for (int k = 0; k < 4; ++k) sc->anchor[k] = sc->info.cam_pos[k] = p->translate[k];
        if (p->config == 5) {
            Rng sr{p->seed ^ 0x5354415253ull};
            sc->num_stars = p->n_stars;
            std::vector<float> hdr, segs;
            for (uint32_t i = 0; i < p->n_stars; ++i) {
                double z = sr.uni(-1, 1), ph = sr.uni(0, 6.283185307179586), rho = std::sqrt(std::max(0.0, 1.0 - z * z));
                double dir[3] = {rho * std::cos(ph), rho * std::sin(ph), z}, b[3];
                sr.ball(b);
                double temp = std::exp(sr.uni(std::log(2000.0), std::log(40000.0)));
                double inten = 1000.0 * 1000.0 * 2e-4 * std::exp(sr.normal());
                V3f beta((float)(0.01 * b[0]), (float)(0.01 * b[1]), (float)(0.01 * b[2]));
                V4f u = four_velocity(beta);
                float tf = (float)temp, inf = (float)inten;
                hdr.insert(hdr.end(), {tf, color_norm(tf, inf), fbits(i), fbits(1u)});
                segs.insert(segs.end(), {0.0f, (float)(1000.0 * dir[0]), (float)(1000.0 * dir[1]), (float)(1000.0 * dir[2]),
                                         u.t, u.x, u.y, u.z, -1e30f, 1e30f, 0.0f, 0.0f});
            }
            sc->stars = hdr;
            sc->stars.insert(sc->stars.end(), segs.begin(), segs.end());
            sc->info.cam_rapidity[0] = 0.8;
            sc->info.cam_rapidity[1] = -0.3;
            sc->info.cam_rapidity[2] = 0.5;
        }
    }
    // Extrude on worker threads; bodies are concatenated in order afterwards.
    std::vector<char> rok(jobs.size(), 1);
    sc->tube_recs.resize(jobs.size());
    {
        std::atomic<size_t> next{0};
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < std::min<size_t>(threads, jobs.size()); ++t)
            pool.emplace_back([&] {
                for (size_t j; (j = next.fetch_add(1)) < jobs.size();) rok[j] = jobs[j](per_body[j], sc->tube_recs[j]) ? 1 : 0;
            });
        for (auto& th : pool) th.join();
    }
    for (auto& rec : sc->tube_recs)
        sc->tubes.push_back(SrTube{rec.verts.data(), (uint32_t)(rec.verts.size() / 3), (uint32_t)rec.tris.size(),
                                   rec.tris.data(), rec.samples.data(), (uint32_t)rec.samples.size(), rec.mat, nullptr});
    sc->info.rindler_ok = 1;
    for (char c : rok) if (!c) sc->info.rindler_ok = 0;
    size_t n = 0;
    for (auto& v : per_body) n += v.size();
    std::vector<Tet> tets;
    tets.reserve(n);
    for (auto& v : per_body) { tets.insert(tets.end(), v.begin(), v.end()); std::vector<Tet>().swap(v); }

    sc->boxes.resize(8 * n);
    for (size_t i = 0; i < n; ++i) {
        put4(&sc->boxes[8 * i], tets[i].box.lo);
        put4(&sc->boxes[8 * i + 4], tets[i].box.hi);
    }
    // BVH.
    std::vector<Ref> refs(n);
    for (size_t i = 0; i < n; ++i) refs[i] = {tets[i].box, (tets[i].box.lo + tets[i].box.hi) * 0.5f, (uint32_t)i};
    unsigned sd = 0;
    while ((1u << sd) < threads * 4) ++sd;
    std::atomic<uint32_t> median{0};
    Builder bld{sd, &median};
    std::vector<Node> nodes = n ? bld.build_sub(refs.data(), n, 0, 0) : std::vector<Node>();
    sc->info.median_splits = median.load();
    sc->nodes.resize(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        SrGpuNode& g = sc->nodes[i];
        put4(g.min, nodes[i].box.lo);
        put4(g.max, nodes[i].box.hi);
        g.right_or_first = nodes[i].right_or_first;
        g.count = nodes[i].count;
        g.left = nodes[i].left;
        g.pad = 0;
        if (g.count > sc->info.max_leaf) sc->info.max_leaf = g.count;
    }
    sc->geoms.resize(n);
    sc->attrs.resize(n);
    sc->order.resize(n);
    for (size_t i = 0; i < n; ++i) {
        sc->order[i] = refs[i].index;
        sc->geoms[i] = tets[refs[i].index].g;
        sc->attrs[i] = tets[refs[i].index].a;
    }
    sc->mats = common_materials();
    // Tree depth.
    uint32_t depth = 0;
    if (!sc->nodes.empty()) {
        std::vector<std::pair<uint32_t, uint32_t>> st{{0u, 1u}};
        while (!st.empty()) {
            auto [i, d] = st.back();
            st.pop_back();
            depth = std::max(depth, d);
            if (sc->nodes[i].count == 0) { st.push_back({sc->nodes[i].left, d + 1}); st.push_back({sc->nodes[i].right_or_first, d + 1}); }
        }
    }
    sc->info.bvh_depth = depth;
    for (int k = 0; k < 4; ++k) sc->info.anchor[k] = sc->anchor[k];
    sc->info.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    *out = sc.release();
    return SR_OK;
}

extern "C" void sr_scene_free(sr_scene* s) { delete s; }

extern "C" sr_status sr_bvh_build_host(const float* boxes, uint32_t n, uint32_t threads, SrGpuNode* nodes,
                                       uint32_t nodes_cap, uint32_t* order, uint32_t* num_nodes,
                                       uint32_t* median_splits) {
    if ((n && (!boxes || !nodes || !order)) || !num_nodes) return SR_ERR_INVALID_ARGUMENT;
    if (n && (uint64_t)nodes_cap < 2ull * n - 1) return SR_ERR_INVALID_ARGUMENT;
    std::vector<Ref> refs(n);
    for (uint32_t i = 0; i < n; ++i) {
        Box b;
        b.lo = V4f(boxes[8 * i], boxes[8 * i + 1], boxes[8 * i + 2], boxes[8 * i + 3]);
        b.hi = V4f(boxes[8 * i + 4], boxes[8 * i + 5], boxes[8 * i + 6], boxes[8 * i + 7]);
        refs[i] = {b, (b.lo + b.hi) * 0.5f, i};
    }
    unsigned sd = 0;
    while ((1u << sd) < std::max(1u, threads) * 4) ++sd;
    std::atomic<uint32_t> median{0};
    Builder bld{sd, &median};
    std::vector<Node> out = n ? bld.build_sub(refs.data(), n, 0, 0) : std::vector<Node>();
    for (size_t i = 0; i < out.size(); ++i) {
        SrGpuNode& g = nodes[i];
        put4(g.min, out[i].box.lo);
        put4(g.max, out[i].box.hi);
        g.right_or_first = out[i].right_or_first;
        g.count = out[i].count;
        g.left = out[i].left;
        g.pad = 0;
    }
    for (uint32_t i = 0; i < n; ++i) order[i] = refs[i].index;
    *num_nodes = (uint32_t)out.size();
    if (median_splits) *median_splits = median.load();
    return SR_OK;
}

extern "C" sr_status sr_scene_desc(const sr_scene* s, SrSceneDesc* d) {
    if (!s || !d) return SR_ERR_INVALID_ARGUMENT;
    std::memset(d, 0, sizeof(*d));
    d->nodes = s->nodes.data();
    d->num_nodes = (uint32_t)s->nodes.size();
    d->num_prims = (uint32_t)s->geoms.size();
    d->geoms = s->geoms.data();
    d->attrs = s->attrs.data();
    d->materials = s->mats.data();
    d->num_materials = (uint32_t)s->mats.size();
    d->num_stars = s->num_stars;
    d->stars = s->stars.empty() ? nullptr : s->stars.data();
    d->num_star_vec4 = s->stars.size() / 4;
    d->light_pos[0] = 0.0f;
    d->light_pos[1] = 0.0f;
    d->light_pos[2] = 50.0f;
    d->light_pos[3] = 0.0f;
    d->leaf_to_orig = s->order.data();
    d->anchor = s->anchor;
    return SR_OK;
}

extern "C" sr_status sr_scene_boxes(const sr_scene* s, const float** boxes) {
    if (!s || !boxes) return SR_ERR_INVALID_ARGUMENT;
    *boxes = s->boxes.empty() ? nullptr : s->boxes.data();
    return SR_OK;
}

extern "C" sr_status sr_scene_tubes(const sr_scene* s, const SrTube** tubes, uint32_t* num_tubes) {
    if (!s || !tubes || !num_tubes) return SR_ERR_INVALID_ARGUMENT;
    *tubes = s->tubes.empty() ? nullptr : s->tubes.data();
    *num_tubes = (uint32_t)s->tubes.size();
    return SR_OK;
}

extern "C" sr_status sr_scene_info(const sr_scene* s, SrSynthInfo* out) {
    if (!s || !out) return SR_ERR_INVALID_ARGUMENT;
    *out = s->info;
    return SR_OK;
}

extern "C" sr_status sr_observers_synth(uint64_t seed, uint32_t n, SrObserverDraw* out) {
    if (!out && n) return SR_ERR_INVALID_ARGUMENT;
    Rng r{seed ^ 0x4F4253ull};
    const uint32_t RES[4][2] = {{320, 200}, {640, 400}, {1280, 800}, {1920, 1200}};
    for (uint32_t i = 0; i < n; ++i) {
        SrObserverDraw& o = out[i];
        uint32_t ri = std::min<uint32_t>(3, (uint32_t)(r.u01() * 4.0));
        o.width = RES[ri][0];
        o.height = RES[ri][1];
        o.pad = 0;
        o.pos[0] = r.uni(-50, 0);
        double x[3];
        r.ball(x);
        for (int k = 0; k < 3; ++k) o.pos[1 + k] = 30.0 * x[k];
        r.ball(x);
        for (int k = 0; k < 3; ++k) o.rapidity[k] = 3.0 * x[k];
        o.slice_mode = r.u01() < 0.5 ? 0u : 1u;
    }
    return SR_OK;
}
