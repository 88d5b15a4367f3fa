// TEST INFRASTRUCTURE ONLY — pins the CPU oracle to the reference's own known-answer tests.
// Each check restates a #[test] of the reference with its tolerance; the program prints one
// line per test and exits non-zero if any fails. Built and run by tests/test_oracle_kat.py.
#include <cstdio>
#include <string>

#include "oracle_scenes.hpp"

using namespace orc;

static int g_fail = 0;
static std::string g_test;
#define CHECK(cond)                                                                          \
    do {                                                                                     \
        if (!(cond)) {                                                                       \
            std::printf("  check failed in %s: %s (line %d)\n", g_test.c_str(), #cond, __LINE__); \
            ok = false;                                                                      \
        }                                                                                    \
    } while (0)
#define TEST(name) static bool name()
#define RUN(name)                                              \
    do {                                                       \
        g_test = #name;                                        \
        bool r = name();                                       \
        std::printf("%s %s\n", r ? "PASS" : "FAIL", #name);    \
        if (!r) ++g_fail;                                      \
    } while (0)

using F = float;
using V3f = V3<F>;
using V4f = V4<F>;

// minkowski.rs:615-626
TEST(cross4_orthogonality) {
    bool ok = true;
    V4f u(1.2f, -0.4f, 0.7f, 2.1f), v(-0.3f, 1.5f, 0.2f, -1.1f), w(0.8f, 0.1f, -1.9f, 0.5f);
    V4f n = V4f::cross4(u, v, w);
    CHECK(n.elen() > 0.1f);
    CHECK(std::fabs(u.edot(n)) < 1e-5f);
    CHECK(std::fabs(v.edot(n)) < 1e-5f);
    CHECK(std::fabs(w.edot(n)) < 1e-5f);
    return ok;
}

// minkowski.rs:628-657
TEST(tetrad_orthonormality_and_null_rays) {
    bool ok = true;
    Tetrad<F> t = Tetrad<F>::from_beta(V3f(0.6f, -0.3f, 0.5f));
    t.rotate_local(0.4f, -0.25f, 0.1f);
    t.boost_local(V3f(0.2f, 0.1f, 0.8f));
    CHECK(std::fabs(t.e[0].mnorm_sq() + 1.0f) < 1e-5f);
    for (int a = 1; a <= 3; ++a) {
        CHECK(std::fabs(t.e[a].mnorm_sq() - 1.0f) < 1e-5f);
        CHECK(std::fabs(t.e[0].mdot(t.e[a])) < 1e-5f);
        for (int b = a + 1; b <= 3; ++b) CHECK(std::fabs(t.e[a].mdot(t.e[b])) < 1e-5f);
    }
    V4f vl(2.3f, -1.1f, 0.7f, 3.4f);
    V4f rec = t.world_to_local(t.local_to_world(vl));
    CHECK(std::fabs(rec.t - vl.t) < 1e-5f && std::fabs(rec.x - vl.x) < 1e-5f);
    CHECK(std::fabs(rec.y - vl.y) < 1e-5f && std::fabs(rec.z - vl.z) < 1e-5f);
    V4f k = t.past_light_ray_direction(V3f(0.3f, -0.4f, 1.0f));
    CHECK(std::fabs(k.mnorm_sq()) < 1e-5f);
    CHECK(k.t < 0.0f);
    return ok;
}

// minkowski.rs:659-691
TEST(relativistic_aberration_formula) {
    bool ok = true;
    F beta = 0.75f;
    Tetrad<F> t = Tetrad<F>::from_beta(V3f(0, 0, beta));
    for (F deg : {0.0f, 30.0f, 60.0f, 90.0f, 120.0f, 150.0f, 180.0f}) {
        F th = deg * (C<F>::PI / 180.0f);
        V4f kl(-1.0f, std::sin(th), 0.0f, std::cos(th));
        V4f ko = t.world_to_local(kl);
        F c = rest_frame_cos(kl, t.e[3], t.e[0]);
        F expected = (std::cos(th) + beta) / (1.0f + beta * std::cos(th));
        CHECK(std::fabs(c - expected) < 1e-5f);
        CHECK(std::fabs(ko.spatial().normalized().z - expected) < 1e-5f);
    }
    return ok;
}

// mesh4d.rs:1095-1125
TEST(worldtube_decided_at_follows_steps) {
    bool ok = true;
    auto mesh = Mesh3D<F>::cube(V3f(0.5f, 0.5f, 0.5f));
    auto samples = sample_inertial_worldline<F>(V3f(), V3f(0.3f, 0, 0), 0.0f, 4.0f, 2);
    CHECK(samples.size() == 3);
    std::vector<Simplex<F>> st;
    extend_worldtube_simplices<F>(st, mesh, samples, (const F*)nullptr, 0);
    for (auto& s : st) for (int i = 0; i < 4; ++i) CHECK(s.decided_at[i] == DECIDED_AT_STATIC);
    F dec[3] = {10, 20, 30};
    std::vector<Simplex<F>> tube;
    extend_worldtube_simplices<F>(tube, mesh, samples, dec, 0);
    CHECK(tube.size() == st.size());
    bool seen[2] = {false, false};
    for (auto& s : tube) {
        F lo = INFINITY, hi = -INFINITY;
        for (int i = 0; i < 4; ++i) { lo = std::fmin(lo, s.decided_at[i]); hi = std::fmax(hi, s.decided_at[i]); }
        int step = lo == 10.0f ? 0 : 1;
        CHECK(lo == dec[step] && hi == dec[step + 1]);
        seen[step] = true;
        std::array<F, 4> b = {0.1f, 0.2f, 0.3f, 0.4f};
        auto h = s.interpolate_hit(1.0f, s.g.v0, b);
        F e = 0;
        for (int i = 0; i < 4; ++i) e += s.decided_at[i] * b[i];
        CHECK(std::fabs(h.decided_at - e) < 1e-4f);
    }
    CHECK(seen[0] && seen[1]);
    return ok;
}

// mesh4d.rs:1127-1160
template <class T> bool ray_simplex_intersection_t() {
    bool ok = true;
    std::array<V4<T>, 4> v = {V4<T>(0, 0, 0, 0), V4<T>(1, 0, 0, 0), V4<T>(0, 1, 0, 0), V4<T>(0, 0, 1, 0)};
    Simplex<T> s;
    bool made = Simplex<T>::make(v, {{{0, 0}, {1, 0}, {0, 1}, {1, 1}}},
                                 {V3<T>(1, 0, 0), V3<T>(1, 0, 0), V3<T>(0, 1, 0), V3<T>(0, 0, 1)}, {0, 1, 0, 0},
                                 {{{0, 0}, {0, 0}, {0, 0}, {0, 0}}}, {1, 1}, V4<T>(0, 0, 0, 1), V4<T>(1, 0, 0, 0), 0, &s);
    CHECK(made);
    HitRecord<T> h;
    bool hit = s.intersect(V4<T>(T(0.2), T(0.2), T(0.2), T(2.0)), V4<T>(0, 0, 0, -1), T(0), T(10), &h);
    CHECK(hit);
    if (!hit) return false;
    CHECK(std::fabs(h.lambda - T(2)) < T(1e-5));
    CHECK(std::fabs(h.tet_bary[1] - T(0.2)) < T(1e-5));
    CHECK(std::fabs(h.tet_bary[2] - T(0.2)) < T(1e-5));
    CHECK(std::fabs(h.tet_bary[3] - T(0.2)) < T(1e-5));
    return ok;
}
TEST(ray_simplex4d_intersection) { return ray_simplex_intersection_t<float>() && ray_simplex_intersection_t<double>(); }

// mesh4d.rs:1162-1192
template <class T> bool length_contraction_t() {
    bool ok = true;
    auto cube = Mesh3D<T>::cube(V3<T>(1, 1, 1));
    auto samples = sample_inertial_worldline<T>(V3<T>(), V3<T>(T(0.8), 0, 0), T(-20), T(20), 4);
    std::vector<Simplex<T>> s;
    extend_worldtube_simplices<T>(s, cube, samples, (const T*)nullptr, 0);
    T mn = INFINITY, mx = -INFINITY;
    for (auto& x : s) {
        HitRecord<T> h;
        if (x.intersect(V4<T>(0, -5, T(0.1), T(0.1)), V4<T>(0, 1, 0, 0), T(0), T(100), &h)) {
            mn = std::fmin(mn, h.event.x);
            mx = std::fmax(mx, h.event.x);
        }
    }
    CHECK(std::fabs((mx - mn) - T(1.2)) < T(1e-4));
    return ok;
}
TEST(emergent_length_contraction_in_worldtube) { return length_contraction_t<float>() && length_contraction_t<double>(); }

// mesh4d.rs:1194-1241
TEST(thomas_precession_one_orbit) {
    bool ok = true;
    double beta = 0.80, gamma = 1.0 / std::sqrt(1.0 - beta * beta), radius = 4.0, omega = beta / radius;
    double period = 2.0 * M_PI / omega;
    auto samples = sample_accelerated_worldline<F>(
        [&](double t) { return Pos3d{radius * std::cos(omega * t), 0.0, radius * std::sin(omega * t)}; }, 0.0f,
        (F)period, 180, nullptr);
    Tetrad<F> t0 = samples.front().tetrad, t1 = samples.back().tetrad;
    t0.boost_to(V4f(1, 0, 0, 0));
    t1.boost_to(V4f(1, 0, 0, 0));
    F a0 = std::atan2(t0.e[1].z, t0.e[1].x), a1 = std::atan2(t1.e[1].z, t1.e[1].x);
    F measured = rem_euclid(a0 - a1, C<F>::TAU);
    F expected = (F)std::fmod((gamma - 1.0) * 2.0 * M_PI, 2.0 * M_PI);
    CHECK(std::fabs(measured - expected) < 5e-3f);
    return ok;
}

// mesh4d.rs:1243-1322 (with sync_proper_time_at, mesh4d.rs:1056-1087)
template <class T> void sync_proper_time_at(std::vector<WorldlineSample<T>>& s, T t_sync) {
    if (s.empty()) return;
    T tau = s[0].proper_time;
    V3<T> phi = s[0].phi;
    if (t_sync <= s[0].center.t) {
    } else if (t_sync >= s.back().center.t) {
        tau = s.back().proper_time;
        phi = s.back().phi;
    } else {
        for (size_t i = 0; i + 1 < s.size(); ++i)
            if (t_sync >= s[i].center.t && t_sync <= s[i + 1].center.t) {
                T dt = std::fmax(s[i + 1].center.t - s[i].center.t, T(1e-6));
                T frac = (t_sync - s[i].center.t) / dt;
                tau = s[i].proper_time + frac * (s[i + 1].proper_time - s[i].proper_time);
                phi = s[i].phi + (s[i + 1].phi - s[i].phi) * frac;
                break;
            }
    }
    for (auto& x : s) { x.proper_time -= tau; x.phi -= phi; }
}
TEST(born_rigid_front_back_proper_time_offset) {
    bool ok = true;
    double beta_max = 0.80;
    F expected_phi = (F)std::atanh(beta_max);
    double k = M_PI / 20.0;
    auto samples = sample_accelerated_worldline<F>(
        [&](double t) {
            double tc = std::min(20.0, std::max(0.0, t));
            return Pos3d{beta_max * (0.5 * tc - std::sin(2.0 * k * tc) / (4.0 * k)), 0.0, 0.0};
        },
        0.0f, 20.0f, 100, nullptr);
    sync_proper_time_at<F>(samples, 0.0f);
    const auto& mid = samples[50];
    CHECK(std::fabs(mid.phi.x - expected_phi) < 2e-3f);
    CHECK(std::fabs(samples.back().phi.x) < 2e-3f);
    auto cube = Mesh3D<F>::cube(V3f(1, 1, 1));
    std::vector<WorldlineSample<F>> part(samples.begin() + 49, samples.begin() + 52);
    std::vector<Simplex<F>> s;
    extend_worldtube_simplices<F>(s, cube, part, (const F*)nullptr, 0);
    for (F xl : {-0.75f, -0.25f, 0.25f, 0.75f}) {
        V4f o = mid.center + mid.tetrad.local_spatial_to_world(V3f(xl, 0.2f, -3.0f));
        V4f d = mid.tetrad.local_spatial_to_world(V3f(0, 0, 1));
        bool found = false;
        HitRecord<F> best;
        for (auto& x : s) {
            HitRecord<F> h;
            if (x.intersect(o, d, 0.0f, 2.5f, &h) && (!found || h.lambda < best.lambda)) { best = h; found = true; }
        }
        CHECK(found);
        if (!found) continue;
        CHECK(std::fabs(best.uvs_u - 2.0f) < 1e-4f);
        CHECK(std::fabs(best.uvs_v - 2.0f) < 1e-4f);
        F central = best.proper_time - (best.uv_u - 0.5f) * best.grad_u - (best.uv_v - 0.5f) * best.grad_v;
        CHECK(std::fabs(central - mid.proper_time) < 1e-3f);
    }
    return ok;
}

// star.rs:329-336
TEST(white_point_is_white_and_doppler_shifts_color) {
    bool ok = true;
    V3f w = blackbody_rgb<F>(WHITE_POINT_K);
    CHECK(std::fabs(w.x - 1) < 1e-5f && std::fabs(w.y - 1) < 1e-5f && std::fabs(w.z - 1) < 1e-5f);
    V3f red = blackbody_rgb<F>(3000.0f), blue = blackbody_rgb<F>(15000.0f);
    CHECK(red.x > red.z && blue.z > blue.x);
    return ok;
}

// star.rs:338-350
TEST(past_cone_event_is_null_and_in_the_past) {
    bool ok = true;
    auto star = PointStar<F>::moving(V3f(3, 1, -4), V3f(0.5f, 0, 0.3f), 5000, 1);
    V4f o(7, 0.5f, 0, 0), e0(1, 0, 0, 0), d, u;
    CHECK(worldline_cone_event(star, o, e0, -1.0f, &d, &u));
    CHECK(std::fabs(d.mnorm_sq()) < 1e-3f && d.t < 0);
    CHECK(worldline_cone_event(star, o, e0, 1.0f, &d, &u));
    CHECK(std::fabs(d.mnorm_sq()) < 1e-3f && d.t > 0);
    CHECK(worldline_cone_event(star, o, e0, 0.0f, &d, &u));
    CHECK(std::fabs(d.t) < 1e-4f);
    return ok;
}

static V3f star_light1(const PointStar<F>& s, const V4f& dir, F spread, F lmax) {
    std::vector<PointStar<F>> v{s};
    std::vector<F> cn{color_norm(s)};
    return star_light<F>(v, cn, V4f(), dir, V4f(1, 0, 0, 0), -1.0f, 0.0f, spread, lmax);
}

// star.rs:352-376
TEST(star_flux_is_conserved_across_subpixel_positions) {
    bool ok = true;
    F pitch = 0.01f, r = 20.0f;
    Tetrad<F> t = Tetrad<F>::rest();
    for (auto off : {std::pair<F, F>{0, 0}, {0.3f, 0.1f}, {0.5f, 0.5f}, {0.77f, 0.21f}}) {
        auto star = PointStar<F>::at_rest(V3f(off.first * pitch * r, off.second * pitch * r, r), WHITE_POINT_K, 1.0f);
        F flux = 0;
        for (int j = -6; j <= 6; ++j)
            for (int i = -6; i <= 6; ++i) {
                F sx = (F)i * pitch, sy = (F)j * pitch;
                V4f dir = t.past_light_ray_direction(V3f(sx, sy, 1));
                F inv_len = 1.0f / std::sqrt(sx * sx + sy * sy + 1.0f);
                F spread = pitch * inv_len * std::sqrt(inv_len);
                V3f l = star_light1(star, dir, spread, 1e30f);
                flux += luminance(l) * spread * spread;
            }
        F expected = 1.0f / (r * r);
        CHECK(std::fabs(flux / expected - 1.0f) < 0.01f);
    }
    return ok;
}

// star.rs:378-401
TEST(polyline_star_is_found_by_segment_and_ends_at_its_last_event) {
    bool ok = true;
    auto star = PointStar<F>::along({V4f(-30, 5, 0, 0), V4f(2, 5, 0, 0), V4f(6, 5, 2, 0)}, 5000, 1);
    V4f e0(1, 0, 0, 0), d, u;
    CHECK(worldline_cone_event(star, V4f(3, 0, 0, 0), e0, -1.0f, &d, &u));
    CHECK(std::fabs(d.x - 5) < 1e-4f && std::fabs(d.y) < 1e-4f && std::fabs(u.t - 1) < 1e-5f);
    CHECK(worldline_cone_event(star, V4f(9, 0, 0, 0), e0, -1.0f, &d, &u));
    CHECK(d.y > 0 && d.y < 2 && u.y > 0 && std::fabs(d.mnorm_sq()) < 1e-3f);
    CHECK(!worldline_cone_event(star, V4f(20, 0, 0, 0), e0, -1.0f, &d, &u));
    CHECK(!worldline_cone_event(star, V4f(-40, 0, 0, 0), e0, -1.0f, &d, &u));
    return ok;
}

// star.rs:403-411
TEST(star_behind_an_occluder_is_hidden) {
    bool ok = true;
    auto s = PointStar<F>::at_rest(V3f(0, 0, 10), WHITE_POINT_K, 1.0f);
    V4f dir(-1, 0, 0, 1);
    CHECK(luminance(star_light1(s, dir, 0.01f, 1e30f)) > 0);
    CHECK(luminance(star_light1(s, dir, 0.01f, 9.0f)) == 0);
    return ok;
}

// star.rs:413-428
TEST(approaching_star_is_blueshifted_and_brighter) {
    bool ok = true;
    V4f dir(-1, 0, 0, 1);
    V3f a = star_light1(PointStar<F>::at_rest(V3f(0, 0, 10), 5000, 1), dir, 0.01f, 1e30f);
    V3f b = star_light1(PointStar<F>::moving(V3f(0, 0, 10), V3f(0, 0, -0.5f), 5000, 1), dir, 0.01f, 1e30f);
    CHECK(b.z / b.x > a.z / a.x);
    CHECK(luminance(b) > luminance(a));
    return ok;
}

// bloom.rs:131-143
TEST(bloom_conserves_energy_and_spreads_a_point) {
    bool ok = true;
    size_t w = 97, h = 64;
    std::vector<V3f> img(w * h);
    img[30 * w + 40] = V3f::splat(1000.0f);
    bloom_apply(img, w, h);
    F total = 0;
    for (auto& c : img) total += c.x;
    CHECK(std::fabs(total / 1000.0f - 1.0f) < 0.01f);
    CHECK(img[30 * w + 40].x > 900.0f);
    F nearv = img[30 * w + 50].x, farv = img[30 * w + 70].x;
    CHECK(nearv > farv && farv > 1e-4f);
    return ok;
}

// bloom.rs:145-151
TEST(flat_image_is_unchanged) {
    bool ok = true;
    size_t w = 33, h = 20;
    std::vector<V3f> img(w * h, V3f::splat(0.5f));
    bloom_apply(img, w, h);
    for (auto& c : img) CHECK(std::fabs(c.x - 0.5f) < 1e-5f);
    return ok;
}

// renderer.rs:1140-1153
TEST(analytic_decision_age_is_time_ago_plus_distance) {
    bool ok = true;
    V4f o(10, 1, 2, 3), u(1, 0, 0, 0);
    auto at = [&](F dt, F r) { return o + V4f(dt, r, 0, 0); };
    CHECK(std::fabs(analytic_decision_age(at(-3, 4), o, u) - 7.0f) < 1e-5f);
    CHECK(std::fabs(analytic_decision_age(at(1, 3), o, u) - 2.0f) < 1e-5f);
    CHECK(std::fabs(analytic_decision_age(at(2, 2), o, u)) < 1e-5f);
    CHECK(analytic_decision_age(at(3, 1), o, u) < 0);
    return ok;
}

// renderer.rs:1155-1168
TEST(analytic_decision_age_on_past_cone_is_round_trip) {
    bool ok = true;
    Tetrad<F> t = Tetrad<F>::rest();
    t.boost_local(V3f(0.4f, -0.2f, 0.7f));
    t.rotate_local(0.3f, 0.1f, -0.2f);
    V4f o(5, -1, 0.5f, 2);
    for (auto dl : {std::pair<V3f, F>{V3f(0, 0, 1), 3.0f}, {V3f(1, -0.5f, 0.2f), 7.5f}}) {
        V4f ev = o + t.past_light_ray_direction(dl.first) * dl.second;
        CHECK(std::fabs(analytic_decision_age(ev, o, t.e[0]) - 2.0f * dl.second) < 1e-3f);
    }
    return ok;
}

// renderer.rs:1188-1211 (the apply_undecided_haze half)
TEST(haze_covers_every_undecided_cone) {
    bool ok = true;
    std::vector<V4f> origins{V4f(6, 6, 0, 0)};
    V3f base(0.5f, 0.5f, 0.5f);
    auto at = [](F x) { return V4f(10, x, 0, 0); };
    V3f a = apply_undecided_haze(base, at(-1), origins);
    CHECK(a.x == base.x && a.y == base.y && a.z == base.z);
    V3f hz = apply_undecided_haze(base, at(6), origins);
    CHECK(hz.z > hz.x && hz.z > hz.y);
    V3f c = apply_undecided_haze(base, at(11), origins);
    CHECK(c.x == base.x && c.y == base.y && c.z == base.z);
    return ok;
}

// Gamma LUT endpoints and the tone curve (renderer.rs:1102-1129).
TEST(gamma_lut_and_pack) {
    bool ok = true;
    const auto& l = gamma_lut();
    CHECK(l[0] == 0 && l[4095] == 255);
    for (size_t i = 1; i < 4096; ++i) CHECK(l[i] >= l[i - 1]);
    CHECK(pack_rgb(V3f(0, 0, 0)) == 0u);
    CHECK(pack_rgb(V3f(1e9f, 1e9f, 1e9f)) == 0xFFFFFFu);
    return ok;
}

// Configuration sanity: cube scene size matches 64 cubes x 12 tris x 64 steps x 3.
TEST(config1_scene_shape) {
    bool ok = true;
    SynthParams p;
    p.config = 1;
    p.seed = 1;
    auto s = synth_scene<float>(p);
    CHECK(s.scene.bvh.hot.size() == 147456u);
    CHECK(s.rindler_ok);
    CHECK(s.scene.bvh.depth() < 63);
    return ok;
}

int main() {
    RUN(cross4_orthogonality);
    RUN(tetrad_orthonormality_and_null_rays);
    RUN(relativistic_aberration_formula);
    RUN(worldtube_decided_at_follows_steps);
    RUN(ray_simplex4d_intersection);
    RUN(emergent_length_contraction_in_worldtube);
    RUN(thomas_precession_one_orbit);
    RUN(born_rigid_front_back_proper_time_offset);
    RUN(white_point_is_white_and_doppler_shifts_color);
    RUN(past_cone_event_is_null_and_in_the_past);
    RUN(star_flux_is_conserved_across_subpixel_positions);
    RUN(polyline_star_is_found_by_segment_and_ends_at_its_last_event);
    RUN(star_behind_an_occluder_is_hidden);
    RUN(approaching_star_is_blueshifted_and_brighter);
    RUN(bloom_conserves_energy_and_spreads_a_point);
    RUN(flat_image_is_unchanged);
    RUN(analytic_decision_age_is_time_ago_plus_distance);
    RUN(analytic_decision_age_on_past_cone_is_round_trip);
    RUN(haze_covers_every_undecided_cone);
    RUN(gamma_lut_and_pack);
    RUN(config1_scene_shape);
    std::printf("%s: %d failed\n", g_fail ? "FAILED" : "OK", g_fail);
    return g_fail ? 1 : 0;
}
