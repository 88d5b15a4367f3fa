// TEST INFRASTRUCTURE ONLY — part of the CPU oracle used by the parity tests as the checker.
//
// 4D geometry, worldtube extrusion and the 4D BVH, restated from the reference:
//   src/mesh4d.rs:62-212   Aabb4D, SimplexGeom4D::intersect_fast
//   src/mesh4d.rs:312-425  Simplex4D::new, interpolate_hit
//   src/mesh4d.rs:453-505  Mesh3D::cube
//   src/mesh4d.rs:662-854  TubeTriangle, extend_worldtube_simplices (Dompierre prism split)
//   src/mesh4d.rs:912-1087 sample_inertial_worldline, sample_accelerated_worldline,
//                          sync_proper_time_at
//   src/bvh4d.rs:8-13,123-141,287-427  box_measure, build, split (8-bin SAH over 4 axes)
//   src/bvh4d.rs:430-578   safe_inv_dir, trace, is_occluded
#pragma once
#include <atomic>
#include <functional>
#include <future>
#include <numeric>
#include <thread>
#include <utility>
#include <vector>

#include "oracle_select.hpp"
#include "oracle_math.hpp"

namespace orc {

// fn(i) for i in [0, n) on the host's threads (work items taken from a shared counter).
template <class F> void parallel_for(uint32_t n, F&& fn) {
    const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), n));
    std::atomic<uint32_t> next{0};
    auto work = [&] {
        for (uint32_t i; (i = next.fetch_add(1)) < n;) fn(i);
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
}

constexpr float DECIDED_AT_STATIC = -1.0e9f;  // mesh4d.rs:5

enum Pattern : uint32_t { CHECKERBOARD = 0, CLOCK_FACE = 1, LIGHT_CLOCK = 2 };

template <class T> struct Material {  // mesh4d.rs:20-60
    V3<T> base_color, checker_color;
    T emission = 0, grid_scale = 1, wireframe_width = 0;
    Pattern pattern = CHECKERBOARD;
    T cavity_length = 1;
};

template <class T> struct Aabb {  // mesh4d.rs:64-147
    V4<T> min = V4<T>::splat(std::numeric_limits<T>::infinity());
    V4<T> max = V4<T>::splat(-std::numeric_limits<T>::infinity());
    void grow(const V4<T>& p) { min = min.vmin(p); max = max.vmax(p); }
    Aabb unite(const Aabb& o) const { Aabb r; r.min = min.vmin(o.min); r.max = max.vmax(o.max); return r; }
    V4<T> center() const { return (min + max) * T(0.5); }
    V4<T> extent() const { return max - min; }
    bool intersect_ray(const V4<T>& o, const V4<T>& inv, T t_min, T t_max, T* enter) const {
        T t0 = (min.t - o.t) * inv.t, t1 = (max.t - o.t) * inv.t;
        T x0 = (min.x - o.x) * inv.x, x1 = (max.x - o.x) * inv.x;
        T y0 = (min.y - o.y) * inv.y, y1 = (max.y - o.y) * inv.y;
        T z0 = (min.z - o.z) * inv.z, z1 = (max.z - o.z) * inv.z;
        T en = fmax_(fmax_(fmax_(fmax_(t_min, fmin_(t0, t1)), fmin_(x0, x1)), fmin_(y0, y1)), fmin_(z0, z1));
        T ex = fmin_(fmin_(fmin_(fmin_(t_max, fmax_(t0, t1)), fmax_(x0, x1)), fmax_(y0, y1)), fmax_(z0, z1));
        if (ex >= en) { *enter = en; return true; }
        return false;
    }
};

// 80-byte hot record (mesh4d.rs:153-212).
template <class T> struct Geom {
    V4<T> v0, n, b1, b2, b3;
    bool intersect_fast(const V4<T>& o, const V4<T>& d, T t_min, T t_max, T* lam, V4<T>* ev,
                        std::array<T, 4>* bary) const {
        T denom = n.edot(d);
        if (std::fabs(denom) < T(1e-9)) return false;
        T lambda = n.edot(v0 - o) / denom;
        if (lambda <= t_min || lambda >= t_max) return false;
        V4<T> event = o + d * lambda;
        V4<T> q = event - v0;
        const T eps = T(-1e-5);
        T u = b1.edot(q);
        if (u < eps || u > T(1) - eps) return false;
        T v = b2.edot(q);
        if (v < eps || u + v > T(1) - eps) return false;
        T w = b3.edot(q);
        if (w < eps || u + v + w > T(1) - eps) return false;
        T w0 = T(1) - u - v - w;
        *lam = lambda;
        *ev = event;
        *bary = {w0, u, v, w};
        return true;
    }
};

template <class T> struct HitRecord {  // mesh4d.rs:277-308
    T lambda;
    V4<T> event;
    std::array<T, 4> tet_bary;
    V3<T> tri_bary;
    T uv_u, uv_v;
    T proper_time;
    T grad_u, grad_v;
    T uvs_u, uvs_v;
    V4<T> normal, four_vel;
    T decided_at;
    uint32_t material_id;
};

template <class T> struct Simplex {  // mesh4d.rs:217-274
    Geom<T> g;
    T uv_u[4], uv_v[4];
    V3<T> tri_bary[4];
    T tau[4];
    T grad_u[4], grad_v[4];
    T uvs_u, uvs_v;
    V4<T> normal, four_vel;
    T decided_at[4];
    uint32_t material_id;
    Aabb<T> aabb;

    // mesh4d.rs:312-371. Returns false for a degenerate tetrahedron.
    static bool make(const std::array<V4<T>, 4>& verts, const std::array<std::pair<T, T>, 4>& uv,
                     const std::array<V3<T>, 4>& tb, const std::array<T, 4>& pt,
                     const std::array<std::pair<T, T>, 4>& grads, std::pair<T, T> uvs,
                     const V4<T>& normal, const V4<T>& four_vel, uint32_t mat, Simplex* out) {
        V4<T> v0 = verts[0];
        V4<T> e1 = verts[1] - v0, e2 = verts[2] - v0, e3 = verts[3] - v0;
        V4<T> n = V4<T>::cross4(e1, e2, e3);
        T n_len_sq = n.elen_sq();
        if (n_len_sq < T(1e-16)) return false;
        T inv_n_len = T(1) / m_sqrt(n_len_sq);
        V4<T> unit_n = n * inv_n_len;
        V4<T> raw_b1 = V4<T>::cross4(e2, e3, unit_n);
        T d1 = raw_b1.edot(e1);
        V4<T> raw_b2 = V4<T>::cross4(e3, e1, unit_n);
        T d2 = raw_b2.edot(e2);
        V4<T> raw_b3 = V4<T>::cross4(e1, e2, unit_n);
        T d3 = raw_b3.edot(e3);
        if (std::fabs(d1) < T(1e-12) || std::fabs(d2) < T(1e-12) || std::fabs(d3) < T(1e-12)) return false;
        Aabb<T> box;
        for (auto& p : verts) box.grow(p);
        V4<T> eps = V4<T>::splat(T(1e-4));
        box.min -= eps;
        box.max += eps;
        Simplex& s = *out;
        s.g.v0 = v0;
        s.g.n = unit_n;
        s.g.b1 = raw_b1 * (T(1) / d1);
        s.g.b2 = raw_b2 * (T(1) / d2);
        s.g.b3 = raw_b3 * (T(1) / d3);
        for (int i = 0; i < 4; ++i) {
            s.uv_u[i] = uv[i].first;
            s.uv_v[i] = uv[i].second;
            s.tri_bary[i] = tb[i];
            s.tau[i] = pt[i];
            s.grad_u[i] = grads[i].first;
            s.grad_v[i] = grads[i].second;
            s.decided_at[i] = T(DECIDED_AT_STATIC);
        }
        s.uvs_u = uvs.first;
        s.uvs_v = uvs.second;
        s.normal = normal;
        s.four_vel = four_vel;
        s.material_id = mat;
        s.aabb = box;
        return true;
    }

    // mesh4d.rs:382-425.
    HitRecord<T> interpolate_hit(T lambda, const V4<T>& event, const std::array<T, 4>& b) const {
        T w0 = b[0], u = b[1], v = b[2], w = b[3];
        HitRecord<T> h;
        h.lambda = lambda;
        h.event = event;
        h.tet_bary = b;
        h.tri_bary = tri_bary[0] * w0 + tri_bary[1] * u + tri_bary[2] * v + tri_bary[3] * w;
        h.uv_u = uv_u[0] * w0 + uv_u[1] * u + uv_u[2] * v + uv_u[3] * w;
        h.uv_v = uv_v[0] * w0 + uv_v[1] * u + uv_v[2] * v + uv_v[3] * w;
        h.proper_time = tau[0] * w0 + tau[1] * u + tau[2] * v + tau[3] * w;
        h.grad_u = grad_u[0] * w0 + grad_u[1] * u + grad_u[2] * v + grad_u[3] * w;
        h.grad_v = grad_v[0] * w0 + grad_v[1] * u + grad_v[2] * v + grad_v[3] * w;
        h.decided_at = decided_at[0] * w0 + decided_at[1] * u + decided_at[2] * v + decided_at[3] * w;
        h.uvs_u = uvs_u;
        h.uvs_v = uvs_v;
        h.normal = normal;
        h.four_vel = four_vel;
        h.material_id = material_id;
        return h;
    }
    bool intersect(const V4<T>& o, const V4<T>& d, T t_min, T t_max, HitRecord<T>* out) const {
        T lam;
        V4<T> ev;
        std::array<T, 4> b;
        if (!g.intersect_fast(o, d, t_min, t_max, &lam, &ev, &b)) return false;
        *out = interpolate_hit(lam, ev, b);
        return true;
    }
};

struct Tri {
    std::array<uint32_t, 3> idx;
    std::array<std::pair<double, double>, 3> uv;  // converted to T at extrusion
};
template <class T> struct Triangle3D {  // mesh4d.rs:438-443
    std::array<uint32_t, 3> indices;
    std::array<std::pair<T, T>, 3> uv;
    V3<T> normal;
};
template <class T> struct Mesh3D {  // mesh4d.rs:447-611
    std::vector<V3<T>> vertices;
    std::vector<Triangle3D<T>> triangles;

    static Mesh3D cube(const V3<T>& he) {  // mesh4d.rs:454-505
        Mesh3D m;
        for (T z : {-he.z, he.z})
            for (T y : {-he.y, he.y})
                for (T x : {-he.x, he.x}) m.vertices.push_back(V3<T>(x, y, z));
        T ux_y = fmax_(round_(he.x / fmax_(he.y, T(1e-4))), T(1));
        T uz_y = fmax_(round_(he.z / fmax_(he.y, T(1e-4))), T(1));
        T ux_z = fmax_(round_(he.x / fmax_(he.z, T(1e-4))), T(1));
        struct F { std::array<uint32_t, 4> i; V3<T> n; T us, vs; };
        const F faces[6] = {
            {{0, 1, 3, 2}, V3<T>(0, 0, -1), ux_y, T(1)}, {{5, 4, 6, 7}, V3<T>(0, 0, 1), ux_y, T(1)},
            {{4, 0, 2, 6}, V3<T>(-1, 0, 0), uz_y, T(1)}, {{1, 5, 7, 3}, V3<T>(1, 0, 0), uz_y, T(1)},
            {{4, 5, 1, 0}, V3<T>(0, -1, 0), ux_z, T(1)}, {{2, 3, 7, 6}, V3<T>(0, 1, 0), ux_z, T(1)},
        };
        for (const F& f : faces) {
            std::pair<T, T> uv0{0, 0}, uv1{f.us, 0}, uv2{f.us, f.vs}, uv3{0, f.vs};
            m.triangles.push_back({{f.i[0], f.i[1], f.i[2]}, {uv0, uv1, uv2}, f.n});
            m.triangles.push_back({{f.i[0], f.i[2], f.i[3]}, {uv0, uv2, uv3}, f.n});
        }
        return m;
    }
};

template <class T> struct WorldlineSample {  // mesh4d.rs:615-630
    V4<T> center;
    T proper_time;
    V3<T> phi;
    V3<T> proper_accel_local;
    Tetrad<T> tetrad;
};

// mesh4d.rs:912-937. `double` stands in for the reference's f64 throughout.
template <class T>
std::vector<WorldlineSample<T>> sample_inertial_worldline(const V3<T>& pos_at_t0, const V3<T>& beta, T t_min,
                                                          T t_max, size_t steps) {
    Tetrad<T> tetrad = Tetrad<T>::from_beta(beta);
    double inv_gamma = 1.0 / (double)tetrad.gamma();
    std::vector<WorldlineSample<T>> out;
    out.reserve(steps + 1);
    for (size_t i = 0; i <= steps; ++i) {
        double frac = (double)i / (double)steps;
        double t = (double)t_min + frac * (double)(t_max - t_min);
        V3<T> pos = pos_at_t0 + beta * (T)t;
        T tau = (T)(t * inv_gamma);
        out.push_back({V4<T>::from_time_space((T)t, pos), tau, V3<T>(), V3<T>(), tetrad});
    }
    return out;
}

// mesh4d.rs:947-1052. `pos_fn` maps lab time to a position (double precision).
struct Pos3d { double x, y, z; };
template <class T>
std::vector<WorldlineSample<T>> sample_accelerated_worldline(const std::function<Pos3d(double)>& pos_fn, T t_min,
                                                             T t_max, size_t steps, bool* superluminal) {
    std::vector<WorldlineSample<T>> samples;
    samples.reserve(steps + 1);
    const double dt_deriv = 1e-5;
    const size_t SUBSTEPS = 8;
    auto velocity = [&](double t) -> Pos3d {
        Pos3d pm = pos_fn(t - dt_deriv), pp = pos_fn(t + dt_deriv);
        double inv_2h = 0.5 / dt_deriv;
        Pos3d v{(pp.x - pm.x) * inv_2h, (pp.y - pm.y) * inv_2h, (pp.z - pm.z) * inv_2h};
        if (!(v.x * v.x + v.y * v.y + v.z * v.z < 1.0) && superluminal) *superluminal = true;
        return v;
    };
    auto four_vel = [&](double t, V4<T>* u) -> double {
        Pos3d v = velocity(t);
        double b2 = std::min(v.x * v.x + v.y * v.y + v.z * v.z, 0.999999999);
        double inv_gamma = std::sqrt(1.0 - b2);
        double gamma = 1.0 / inv_gamma;
        *u = V4<T>((T)gamma, (T)(gamma * v.x), (T)(gamma * v.y), (T)(gamma * v.z));
        return inv_gamma;
    };
    auto proper_accel_world = [&](double t) -> V4<T> {
        V4<T> u0, um, up;
        double inv_gamma = four_vel(t, &u0);
        four_vel(t - dt_deriv, &um);
        four_vel(t + dt_deriv, &up);
        V4<T> du_dt = (up - um) * (T(0.5) / (T)dt_deriv);
        return du_dt * (T(1) / (T)inv_gamma);
    };
    double t_min_d = (double)t_min;
    double t_span_d = (double)(t_max - t_min);
    Pos3d v0 = velocity(t_min_d);
    Tetrad<T> tetrad = Tetrad<T>::from_beta(V3<T>((T)v0.x, (T)v0.y, (T)v0.z));
    double tau = 0.0;
    V3<T> phi;
    double prev_t = t_min_d;
    for (size_t i = 0; i <= steps; ++i) {
        double frac = (double)i / (double)steps;
        double t = t_min_d + frac * t_span_d;
        if (i > 0) {
            double sub_dt = (t - prev_t) / (double)SUBSTEPS;
            for (size_t s = 0; s < SUBSTEPS; ++s) {
                double ta = prev_t + (double)s * sub_dt;
                double tb = ta + sub_dt;
                double tm = 0.5 * (ta + tb);
                V4<T> ua, um_, ub;
                double inv_ga = four_vel(ta, &ua);
                double inv_gm = four_vel(tm, &um_);
                double inv_gb = four_vel(tb, &ub);
                tau += (sub_dt / 6.0) * (inv_ga + 4.0 * inv_gm + inv_gb);
                V4<T> du = ub - ua;
                V3<T> before = tetrad.world_to_local_spatial(du);
                tetrad.fermi_walker_transport(ub);
                V3<T> after = tetrad.world_to_local_spatial(du);
                phi += (before + after) * T(0.5);
            }
        }
        prev_t = t;
        Pos3d p = pos_fn(t);
        V4<T> a_world = proper_accel_world(t);
        V3<T> a_local = tetrad.world_to_local_spatial(a_world);
        samples.push_back({V4<T>((T)t, (T)p.x, (T)p.y, (T)p.z), (T)tau, phi, a_local, tetrad});
    }
    return samples;
}

// mesh4d.rs:663-718.
template <class T> struct TubeTriangle {
    std::array<uint32_t, 3> indices;
    std::array<V3<T>, 3> p;
    std::array<std::pair<T, T>, 3> uv;
    std::array<V3<T>, 3> bary;
    V3<T> tu, tv, normal;
    TubeTriangle(const Mesh3D<T>& mesh, const Triangle3D<T>& tri) {
        const V3<T> std_bary[3] = {V3<T>(1, 0, 0), V3<T>(0, 1, 0), V3<T>(0, 0, 1)};
        std::array<int, 3> perm = {0, 1, 2};
        std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return tri.indices[a] < tri.indices[b]; });
        for (int k = 0; k < 3; ++k) {
            indices[k] = tri.indices[perm[k]];
            p[k] = mesh.vertices[indices[k]];
            uv[k] = tri.uv[perm[k]];
            bary[k] = std_bary[perm[k]];
        }
        V3<T> pa = p[0], pb = p[1], pc = p[2];
        auto uva = uv[0], uvb = uv[1], uvc = uv[2];
        V3<T> dp1 = pb - pa, dp2 = pc - pa;
        T du1 = uvb.first - uva.first, dv1 = uvb.second - uva.second;
        T du2 = uvc.first - uva.first, dv2 = uvc.second - uva.second;
        T uv_det = du1 * dv2 - dv1 * du2;
        if (std::fabs(uv_det) > T(1e-10)) {
            T inv_det = T(1) / uv_det;
            tu = (dp1 * dv2 - dp2 * dv1) * inv_det;
            tv = (dp2 * du1 - dp1 * du2) * inv_det;
        } else {
            tu = V3<T>();
            tv = V3<T>();
        }
        normal = tri.normal;
    }
};

// mesh4d.rs:721-854. Returns false if a sample crosses its Rindler horizon (the reference
// asserts there).
template <class T>
bool extend_worldtube_simplices(std::vector<Simplex<T>>& out, const Mesh3D<T>& mesh,
                                const std::vector<WorldlineSample<T>>& samples, const T* decided_at,
                                uint32_t material_id) {
    if (samples.size() < 2) return true;
    size_t n_verts = mesh.vertices.size();
    size_t n_steps = samples.size() - 1;
    std::vector<V4<T>> ev;
    ev.reserve(samples.size() * n_verts);
    bool ok = true;
    for (auto& s : samples)
        for (auto& pr : mesh.vertices) {
            T rf = T(1) + s.proper_accel_local.dot(pr);
            if (!(rf > T(0))) ok = false;
            ev.push_back(s.center + s.tetrad.local_spatial_to_world(pr));
        }
    std::vector<TubeTriangle<T>> tris;
    tris.reserve(mesh.triangles.size());
    for (auto& tr : mesh.triangles) tris.emplace_back(mesh, tr);
    out.reserve(out.size() + n_steps * 3 * tris.size());
    for (size_t step = 0; step < n_steps; ++step) {
        const V4<T>* vc = &ev[step * n_verts];
        const V4<T>* vn = &ev[(step + 1) * n_verts];
        const auto& sc = samples[step];
        const auto& sn = samples[step + 1];
        T dec0 = decided_at ? decided_at[step] : T(DECIDED_AT_STATIC);
        T dec1 = decided_at ? decided_at[step + 1] : T(DECIDED_AT_STATIC);
        V4<T> u_raw = sc.tetrad.e[0] + sn.tetrad.e[0];
        T u_norm = m_sqrt(fmax_(-u_raw.mnorm_sq(), T(1e-12)));
        V4<T> u_avg = u_raw * (T(1) / u_norm);
        for (auto& tri : tris) {
            uint32_t ia = tri.indices[0], ib = tri.indices[1], ic = tri.indices[2];
            V4<T> a0 = vc[ia], b0 = vc[ib], c0 = vc[ic], a1 = vn[ia], b1 = vn[ib], c1 = vn[ic];
            V3<T> pa = tri.p[0], pb = tri.p[1], pc = tri.p[2];
            T ta0 = sc.proper_time + pa.dot(sc.phi), tb0 = sc.proper_time + pb.dot(sc.phi),
              tc0 = sc.proper_time + pc.dot(sc.phi);
            T ta1 = sn.proper_time + pa.dot(sn.phi), tb1 = sn.proper_time + pb.dot(sn.phi),
              tc1 = sn.proper_time + pc.dot(sn.phi);
            auto uva = tri.uv[0], uvb = tri.uv[1], uvc = tri.uv[2];
            std::pair<T, T> uvs{tri.tu.length(), tri.tv.length()};
            std::pair<T, T> g0{tri.tu.dot(sc.phi), tri.tv.dot(sc.phi)};
            std::pair<T, T> g1{tri.tu.dot(sn.phi), tri.tv.dot(sn.phi)};
            V3<T> ba = tri.bary[0], bb = tri.bary[1], bc = tri.bary[2];
            V4<T> n4c = sc.tetrad.local_spatial_to_world(tri.normal);
            V4<T> n4n = sn.tetrad.local_spatial_to_world(tri.normal);
            V4<T> n4r = n4c + n4n;
            T n4l = m_sqrt(fmax_(n4r.mnorm_sq(), T(1e-12)));
            V4<T> nrm = n4r * (T(1) / n4l);
            struct Tet {
                std::array<V4<T>, 4> v;
                std::array<std::pair<T, T>, 4> uv;
                std::array<V3<T>, 4> tb;
                std::array<T, 4> tau;
                std::array<std::pair<T, T>, 4> g;
                std::array<T, 4> dec;
            };
            const Tet tets[3] = {
                {{a0, b0, c0, c1}, {uva, uvb, uvc, uvc}, {ba, bb, bc, bc}, {ta0, tb0, tc0, tc1}, {g0, g0, g0, g1},
                 {dec0, dec0, dec0, dec1}},
                {{a0, b0, b1, c1}, {uva, uvb, uvb, uvc}, {ba, bb, bb, bc}, {ta0, tb0, tb1, tc1}, {g0, g0, g1, g1},
                 {dec0, dec0, dec1, dec1}},
                {{a0, a1, b1, c1}, {uva, uva, uvb, uvc}, {ba, ba, bb, bc}, {ta0, ta1, tb1, tc1}, {g0, g1, g1, g1},
                 {dec0, dec1, dec1, dec1}},
            };
            for (const Tet& t : tets) {
                Simplex<T> s;
                if (Simplex<T>::make(t.v, t.uv, t.tb, t.tau, t.g, uvs, nrm, u_avg, material_id, &s)) {
                    for (int i = 0; i < 4; ++i) s.decided_at[i] = t.dec[i];
                    out.push_back(s);
                }
            }
        }
    }
    return ok;
}

// ------------------------------------------------------------------------------------------
// 4D BVH (bvh4d.rs).
// ------------------------------------------------------------------------------------------
template <class T> inline T box_measure(const Aabb<T>& b) {  // bvh4d.rs:8-13
    V4<T> e = b.extent();
    T spatial_sa = e.x * e.y + e.y * e.z + e.z * e.x;
    T temporal_sa = T(0.22) * e.t * (e.x + e.y + e.z);
    return spatial_sa + temporal_sa;
}

template <class T> struct BvhNode {
    Aabb<T> aabb;
    uint32_t right_or_first = 0, count = 0, left = 0;
};

// Traversal statistics for the algorithmic-bytes model.
struct TraceStats {
    uint64_t internal_pops = 0;  // internal nodes popped (two child boxes tested each)
    uint64_t leaf_pops = 0;
    uint64_t tets_tested = 0;
    uint64_t max_stack = 0;
    uint64_t overflow = 0;  // children dropped because the 64-entry stack was full
};

template <class T> struct Bvh {
    std::vector<BvhNode<T>> nodes;
    std::vector<Geom<T>> hot;       // leaf order
    std::vector<uint32_t> order;    // leaf slot -> index into `simplices`
    std::vector<Simplex<T>> simplices;  // build order
    uint32_t median_splits = 0;         // nodes split at the centroid median (bvh4d.rs:418-424)

    struct Ref { Aabb<T> aabb; V4<T> centroid; uint32_t index; };

    // bvh4d.rs:123-141; the serial build gives the same tree as the reference's parallel one
    // (bvh4d.rs:254-279: children are spliced in depth-first order either way).
    static Bvh build(std::vector<Simplex<T>> simplices) {
        Bvh b;
        size_t n = simplices.size();
        std::vector<Ref> refs(n);
        for (size_t i = 0; i < n; ++i) refs[i] = {simplices[i].aabb, simplices[i].aabb.center(), (uint32_t)i};
        std::atomic<uint32_t> med{0};
        if (n > 0) {
            b.nodes.reserve(n);
            build_recursive(b.nodes, refs.data(), refs.size(), 0, 6, &med);
        }
        b.median_splits = med.load();
        b.order.resize(n);
        b.hot.resize(n);
        for (size_t i = 0; i < n; ++i) {
            b.order[i] = refs[i].index;
            b.hot[i] = simplices[refs[i].index].g;
        }
        b.simplices = std::move(simplices);
        return b;
    }
    const Simplex<T>& leaf_simplex(size_t i) const { return simplices[order[i]]; }

    // Large subtrees are built on a second thread into their own arrays and spliced in depth-
    // first order (left subtree, then right), which gives the serial build's array exactly: the
    // two subtrees own disjoint ranges of `refs`.
    static uint32_t build_recursive(std::vector<BvhNode<T>>& nodes, Ref* refs, size_t count, size_t first,
                                    int spawn_depth, std::atomic<uint32_t>* med) {
        uint32_t node_idx = (uint32_t)nodes.size();
        Aabb<T> bounds;
        size_t mid;
        bool leaf = !split(refs, count, &bounds, &mid, med);
        if (leaf) {
            BvhNode<T> nd;
            nd.aabb = bounds;
            nd.right_or_first = (uint32_t)first;
            nd.count = (uint32_t)count;
            nodes.push_back(nd);
            return node_idx;
        }
        BvhNode<T> nd;
        nd.aabb = bounds;
        nd.left = node_idx + 1;
        nodes.push_back(nd);
        if (spawn_depth > 0 && count >= 65536) {
            std::vector<BvhNode<T>> ln, rn;
            auto fl = std::async(std::launch::async, [&] { build_recursive(ln, refs, mid, first, spawn_depth - 1, med); });
            build_recursive(rn, refs + mid, count - mid, first + mid, spawn_depth - 1, med);
            fl.get();
            const uint32_t lbase = node_idx + 1, rbase = lbase + (uint32_t)ln.size();
            for (auto* part : {&ln, &rn}) {
                const uint32_t base = part == &ln ? lbase : rbase;
                for (BvhNode<T> x : *part) {
                    if (x.count == 0) {
                        x.left += base;
                        x.right_or_first += base;
                    }
                    nodes.push_back(x);
                }
            }
            nodes[node_idx].right_or_first = rbase;
            return node_idx;
        }
        build_recursive(nodes, refs, mid, first, 0, med);
        uint32_t right_idx = build_recursive(nodes, refs + mid, count - mid, first + mid, 0, med);
        nodes[node_idx].right_or_first = right_idx;
        return node_idx;
    }

    // bvh4d.rs:307-427. Returns false for a leaf.
    static bool split(Ref* refs, size_t count, Aabb<T>* bounds_out, size_t* mid_out, std::atomic<uint32_t>* med) {
        Aabb<T> bounds, cb;
        for (size_t i = 0; i < count; ++i) {
            bounds = bounds.unite(refs[i].aabb);
            cb.grow(refs[i].centroid);
        }
        *bounds_out = bounds;
        if (count <= 3) return false;
        V4<T> ext = cb.extent();
        const int BINS = 8;
        int best_axis = 0;
        T best_split_pos = 0;
        T best_cost = std::numeric_limits<T>::infinity();
        bool live[4];
        T axis_min[4], inv_ext[4];
        for (int a = 0; a < 4; ++a) {
            live[a] = ext.axis(a) >= T(1e-4);
            axis_min[a] = cb.min.axis(a);
            inv_ext[a] = T(BINS) / ext.axis(a);
        }
        Aabb<T> bin_bounds[4][BINS];
        uint32_t bin_counts[4][BINS] = {};
        for (size_t i = 0; i < count; ++i) {
            const Ref& r = refs[i];
            for (int a = 0; a < 4; ++a) {
                if (!live[a]) continue;
                T c = r.centroid.axis(a);
                uint64_t bi = std::min<uint64_t>(as_usize((c - axis_min[a]) * inv_ext[a]), BINS - 1);
                bin_bounds[a][bi] = bin_bounds[a][bi].unite(r.aabb);
                bin_counts[a][bi] += 1;
            }
        }
        for (int a = 0; a < 4; ++a) {
            if (!live[a]) continue;
            T axis_ext = ext.axis(a);
            Aabb<T> left_box[BINS - 1];
            uint32_t left_cnt[BINS - 1];
            Aabb<T> cur_b;
            uint32_t cur_c = 0;
            for (int i = 0; i < BINS - 1; ++i) {
                cur_b = cur_b.unite(bin_bounds[a][i]);
                cur_c += bin_counts[a][i];
                left_box[i] = cur_b;
                left_cnt[i] = cur_c;
            }
            Aabb<T> right_b;
            uint32_t right_c = 0;
            for (int i = BINS - 2; i >= 0; --i) {
                right_b = right_b.unite(bin_bounds[a][i + 1]);
                right_c += bin_counts[a][i + 1];
                if (left_cnt[i] > 0 && right_c > 0) {
                    T cost = (T)left_cnt[i] * box_measure(left_box[i]) + (T)right_c * box_measure(right_b);
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = a;
                        best_split_pos = axis_min[a] + ((T)(i + 1) / (T)BINS) * axis_ext;
                    }
                }
            }
        }
        if (best_cost == std::numeric_limits<T>::infinity()) {
            T max_e = T(-1);
            for (int a = 0; a < 4; ++a)
                if (ext.axis(a) > max_e) { max_e = ext.axis(a); best_axis = a; }
            if (max_e < T(1e-5)) return false;
            best_split_pos = cb.center().axis(best_axis);
        }
        size_t mid = 0;
        for (size_t i = 0; i < count; ++i)
            if (refs[i].centroid.axis(best_axis) < best_split_pos) { std::swap(refs[i], refs[mid]); ++mid; }
        if (mid == 0 || mid == count) {  // bvh4d.rs:418-424
            mid = count / 2;
            select_nth_unstable(refs, count, mid, [best_axis](const Ref& a, const Ref& b) {
                return a.centroid.axis(best_axis) < b.centroid.axis(best_axis);  // partial_cmp == Less
            });
            if (med) med->fetch_add(1);
        }
        *mid_out = mid;
        return true;
    }

    static V4<T> safe_inv_dir(const V4<T>& d) {  // bvh4d.rs:430-441
        auto inv = [](T v) -> T {
            if (std::fabs(v) > T(1e-12)) return T(1) / v;
            return v >= T(0) ? T(1e12) : T(-1e12);
        };
        return V4<T>(inv(d.t), inv(d.x), inv(d.y), inv(d.z));
    }

    // bvh4d.rs:445-520. Returns the leaf slot of the closest hit or -1; fills lambda/event/bary.
    int64_t trace_raw(const V4<T>& o, const V4<T>& d, T t_min, T t_max, T* lam_out, V4<T>* ev_out,
                      std::array<T, 4>* bary_out, TraceStats* st = nullptr) const {
        if (nodes.empty()) return -1;
        V4<T> inv = safe_inv_dir(d);
        T root_enter;
        if (!nodes[0].aabb.intersect_ray(o, inv, t_min, t_max, &root_enter)) return -1;
        int64_t best = -1;
        uint32_t sn[64];
        T stt[64];
        size_t sp = 1;
        sn[0] = 0;
        stt[0] = root_enter;
        while (sp > 0) {
            --sp;
            uint32_t ni = sn[sp];
            T te = stt[sp];
            if (te >= t_max) continue;
            const BvhNode<T>& node = nodes[ni];
            if (node.count > 0) {
                if (st) st->leaf_pops++;
                size_t first = node.right_or_first, end = first + node.count;
                for (size_t k = first; k < end; ++k) {
                    if (st) st->tets_tested++;
                    T lam;
                    V4<T> ev;
                    std::array<T, 4> b;
                    if (hot[k].intersect_fast(o, d, t_min, t_max, &lam, &ev, &b)) {
                        t_max = lam;
                        best = (int64_t)k;
                        *lam_out = lam;
                        *ev_out = ev;
                        *bary_out = b;
                    }
                }
            } else {
                if (st) st->internal_pops++;
                uint32_t li = node.left, ri = node.right_or_first;
                T tl, tr;
                bool hl = nodes[li].aabb.intersect_ray(o, inv, t_min, t_max, &tl);
                bool hr = nodes[ri].aabb.intersect_ray(o, inv, t_min, t_max, &tr);
                if (hl && hr) {
                    if (sp + 2 <= 64) {
                        if (tl <= tr) { sn[sp] = ri; stt[sp] = tr; sn[sp + 1] = li; stt[sp + 1] = tl; }
                        else { sn[sp] = li; stt[sp] = tl; sn[sp + 1] = ri; stt[sp + 1] = tr; }
                        sp += 2;
                    } else if (st) st->overflow++;
                } else if (hl) {
                    if (sp < 64) { sn[sp] = li; stt[sp] = tl; ++sp; } else if (st) st->overflow++;
                } else if (hr) {
                    if (sp < 64) { sn[sp] = ri; stt[sp] = tr; ++sp; } else if (st) st->overflow++;
                }
                if (st && sp > st->max_stack) st->max_stack = sp;
            }
        }
        return best;
    }

    bool trace(const V4<T>& o, const V4<T>& d, T t_min, T t_max, HitRecord<T>* out, int64_t* slot = nullptr,
               TraceStats* st = nullptr) const {
        T lam;
        V4<T> ev;
        std::array<T, 4> b;
        int64_t k = trace_raw(o, d, t_min, t_max, &lam, &ev, &b, st);
        if (slot) *slot = k;
        if (k < 0) return false;
        *out = leaf_simplex((size_t)k).interpolate_hit(lam, ev, b);
        return true;
    }

    // bvh4d.rs:523-578.
    bool is_occluded(const V4<T>& o, const V4<T>& d, T t_min, T t_max, TraceStats* st = nullptr) const {
        if (nodes.empty()) return false;
        V4<T> inv = safe_inv_dir(d);
        T e;
        if (!nodes[0].aabb.intersect_ray(o, inv, t_min, t_max, &e)) return false;
        uint32_t stack[64];
        size_t sp = 1;
        stack[0] = 0;
        while (sp > 0) {
            --sp;
            const BvhNode<T>& node = nodes[stack[sp]];
            if (node.count > 0) {
                if (st) st->leaf_pops++;
                size_t first = node.right_or_first, end = first + node.count;
                for (size_t k = first; k < end; ++k) {
                    if (st) st->tets_tested++;
                    T lam;
                    V4<T> ev;
                    std::array<T, 4> b;
                    if (hot[k].intersect_fast(o, d, t_min, t_max, &lam, &ev, &b)) return true;
                }
            } else {
                if (st) st->internal_pops++;
                uint32_t li = node.left, ri = node.right_or_first;
                T tmp;
                bool hl = nodes[li].aabb.intersect_ray(o, inv, t_min, t_max, &tmp);
                bool hr = nodes[ri].aabb.intersect_ray(o, inv, t_min, t_max, &tmp);
                if (hr) { if (sp < 64) stack[sp++] = ri; else if (st) st->overflow++; }
                if (hl) { if (sp < 64) stack[sp++] = li; else if (st) st->overflow++; }
            }
        }
        return false;
    }

    uint32_t depth() const {
        if (nodes.empty()) return 0;
        uint32_t best = 0;
        std::vector<std::pair<uint32_t, uint32_t>> st{{0u, 1u}};
        while (!st.empty()) {
            auto [i, dd] = st.back();
            st.pop_back();
            best = std::max(best, dd);
            if (nodes[i].count == 0) {
                st.push_back({nodes[i].left, dd + 1});
                st.push_back({nodes[i].right_or_first, dd + 1});
            }
        }
        return best;
    }
};

}  // namespace orc
