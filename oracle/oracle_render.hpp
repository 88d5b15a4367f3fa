// TEST INFRASTRUCTURE ONLY — part of the CPU oracle used by the parity tests as the checker.
//
// Point stars, bloom and the per-pixel renderer, restated from the reference:
//   src/star.rs:41-286       RayFootprint, planck, blackbody_rgb, segment_cone_crossing,
//                            past_the_cone, worldline_cone_event, star_light
//   src/bloom.rs (all)       level_size, level_offset, downsample, upsample_at, apply
//   src/renderer.rs:43-1134  Camera4D, modes, FrameDynamics, render_frame, shade_hit and every
//                            texture / lighting helper, gamma LUT and pack
//   src/hud.rs:473-532       the 5x7 glyphs the clock readout uses
#pragma once
#include <atomic>
#include <thread>
#include <vector>

#include "oracle_geom.hpp"

namespace orc {

// ------------------------------------------------------------------------------------------
// Stars (star.rs).
// ------------------------------------------------------------------------------------------
constexpr float KERNEL_SIGMA = 0.6f;
constexpr float KERNEL_CUTOFF_SIGMAS = 4.0f;
constexpr float WHITE_POINT_K = 6504.0f;
constexpr float UNBOUNDED = 1e30f;

template <class T> struct StarSegment { V4<T> event, four_velocity; T s_min, s_max; };
template <class T> struct PointStar {
    std::vector<StarSegment<T>> segments;
    T temperature = 0, intensity = 0;
    static PointStar moving(const V3<T>& pos, const V3<T>& beta, T temp, T inten) {  // star.rs:85-93
        PointStar s;
        s.segments.push_back({V4<T>::from_time_space(0, pos), V4<T>::four_velocity_from_beta(beta), T(-UNBOUNDED),
                              T(UNBOUNDED)});
        s.temperature = temp;
        s.intensity = inten;
        return s;
    }
    static PointStar at_rest(const V3<T>& pos, T temp, T inten) { return moving(pos, V3<T>(), temp, inten); }
    static PointStar along(const std::vector<V4<T>>& events, T temp, T inten) {  // star.rs:97-112
        PointStar s;
        for (size_t i = 0; i + 1 < events.size(); ++i) {
            V4<T> d = events[i + 1] - events[i];
            T sl = m_sqrt(fmax_(-d.mnorm_sq(), T(0)));
            if (sl > T(1e-6) && d.t > T(0)) s.segments.push_back({events[i], d * (T(1) / sl), T(0), sl});
        }
        s.temperature = temp;
        s.intensity = inten;
        return s;
    }
};

template <class T> inline T luminance(const V3<T>& c) {  // star.rs:156-158
    return T(0.2126) * c.x + T(0.7152) * c.y + T(0.0722) * c.z;
}
// star.rs:162-166. `lambda_um.powi(5)` has a constant base at every call site, so the compiled
// reference folds it at compile time (LLVM evaluates powi of constants in double precision and
// rounds once); the oracle does the same.
template <class T> inline T pow5_const(T x) { return (T)std::pow((double)x, 5.0); }
template <class T> inline T planck(T lambda_um, T temperature) {
    T x = fmin_(T(14388.0) / (lambda_um * fmax_(temperature, T(1))), T(80));
    return T(1) / (pow5_const(lambda_um) * (m_exp(x) - T(1)));
}
template <class T> inline V3<T> blackbody_rgb(T temperature) {  // star.rs:171-180
    const T R = T(0.610), G = T(0.550), B = T(0.465), W = T(WHITE_POINT_K);
    return V3<T>(planck(R, temperature) / planck(R, W), planck(G, temperature) / planck(G, W),
                 planck(B, temperature) / planck(B, W));
}
template <class T> inline T color_norm(const PointStar<T>& s) {  // star.rs:117-124
    T lum = luminance(blackbody_rgb(s.temperature));
    return lum > T(0) ? s.intensity / lum : T(0);
}
template <class T>
inline T segment_cone_crossing(const StarSegment<T>& seg, const V4<T>& origin, const V4<T>& e0, T cone) {
    V4<T> d0 = seg.event - origin;
    V4<T> u = seg.four_velocity;
    if (cone == T(0)) {
        T tau0 = -d0.mdot(e0);
        T gamma = -u.mdot(e0);
        return -tau0 / gamma;
    }
    T a = d0.mnorm_sq();
    T b = d0.mdot(u);
    T sq = m_sqrt(fmax_(b * b + a, T(0)));
    if (cone < T(0)) return b > T(0) ? -a / (b + sq) : b - sq;
    return b < T(0) ? -a / (b - sq) : b + sq;
}
template <class T> inline T past_the_cone(const V4<T>& event, const V4<T>& origin, const V4<T>& e0, T cone) {
    V4<T> d = event - origin;
    T tau = -d.mdot(e0);
    if (cone == T(0)) return tau;
    T rho = m_sqrt(fmax_(d.mnorm_sq() + tau * tau, T(0)));
    return tau - cone * rho;
}
template <class T>
inline bool worldline_cone_event(const PointStar<T>& star, const V4<T>& origin, const V4<T>& e0, T cone,
                                 V4<T>* d_out, V4<T>* u_out) {  // star.rs:228-235
    const auto& segs = star.segments;
    size_t lo = 0, hi = segs.size();  // partition_point
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (past_the_cone(segs[mid].event, origin, e0, cone) <= T(0)) lo = mid + 1;
        else hi = mid;
    }
    size_t idx = std::max<size_t>(lo, 1) - 1;
    if (idx >= segs.size()) return false;
    const auto& seg = segs[idx];
    T s = segment_cone_crossing(seg, origin, e0, cone);
    if (!(s >= seg.s_min && s <= seg.s_max)) return false;
    *d_out = seg.event - origin + seg.four_velocity * s;
    *u_out = seg.four_velocity;
    return true;
}
// star.rs:240-286. `cn` holds each star's color_norm (precomputed, as the packed header does).
template <class T>
V3<T> star_light(const std::vector<PointStar<T>>& stars, const std::vector<T>& cn, const V4<T>& origin,
                 const V4<T>& dir, const V4<T>& e0, T cone, T fp_width, T fp_spread, T lambda_max) {
    V4<T> n = dir - e0 * cone;
    V3<T> total;
    for (size_t i = 0; i < stars.size(); ++i) {
        V4<T> d, u;
        if (!worldline_cone_event(stars[i], origin, e0, cone, &d, &u)) continue;
        T tau = -d.mdot(e0);
        V4<T> r = d + e0 * (-tau);
        T along = r.mdot(n);
        if (along <= T(0) || along >= lambda_max) continue;
        V4<T> perp = r - n * along;
        T d2 = fmax_(perp.mnorm_sq(), T(0));
        T sigma = T(KERNEL_SIGMA) * (fp_width + fp_spread * along);
        T cut = T(KERNEL_CUTOFF_SIGMAS) * sigma;
        if (d2 >= cut * cut) continue;
        T inv_2s2 = T(1) / (T(2) * sigma * sigma);
        T kernel = m_exp(-d2 * inv_2s2) * inv_2s2 * C<T>::FRAC_1_PI;
        T doppler = T(1);
        if (cone < T(0)) {
            T lambda = m_sqrt(fmax_(r.mnorm_sq(), T(0)));
            T du = d.mdot(u);
            if (du > T(0)) doppler = lambda / du;
        }
        total += blackbody_rgb(stars[i].temperature * doppler) * (cn[i] * kernel);
    }
    return total;
}

// ------------------------------------------------------------------------------------------
// Bloom (bloom.rs).
// ------------------------------------------------------------------------------------------
constexpr size_t BLOOM_LEVELS = 6;
constexpr float BLOOM_STRENGTH = 0.04f;
inline std::pair<size_t, size_t> level_size(size_t w, size_t h, size_t k) {
    for (size_t i = 0; i < k; ++i) { w = (w + 1) / 2; h = (h + 1) / 2; }
    return {w, h};
}
inline size_t level_offset(size_t w, size_t h, size_t k) {
    size_t off = 0;
    for (size_t i = 0; i < k; ++i) { auto [a, b] = level_size(w, h, i); off += a * b; }
    return off;
}
inline size_t pyramid_len(size_t w, size_t h) { return level_offset(w, h, BLOOM_LEVELS + 1); }

template <class T> void bloom_downsample(std::vector<V3<T>>& pyr, size_t width, size_t height, size_t k) {
    const T DW[4] = {T(0.125), T(0.375), T(0.375), T(0.125)};
    auto [sw, sh] = level_size(width, height, k - 1);
    auto [dw, dh] = level_size(width, height, k);
    size_t so = level_offset(width, height, k - 1), dof = level_offset(width, height, k);
    for (size_t y = 0; y < dh; ++y)
        for (size_t x = 0; x < dw; ++x) {
            V3<T> acc;
            for (int j = 0; j < 4; ++j) {
                int64_t syi = std::clamp<int64_t>(2 * (int64_t)y - 1 + j, 0, (int64_t)sh - 1);
                V3<T> row;
                for (int i = 0; i < 4; ++i) {
                    int64_t sxi = std::clamp<int64_t>(2 * (int64_t)x - 1 + i, 0, (int64_t)sw - 1);
                    row += pyr[so + (size_t)syi * sw + (size_t)sxi] * DW[i];
                }
                acc += row * DW[j];
            }
            pyr[dof + y * dw + x] = acc;
        }
}
template <class T> V3<T> upsample_at(const V3<T>* coarse, size_t cw, size_t ch, size_t x, size_t y) {
    auto taps = [](size_t i, size_t n) -> std::pair<size_t, size_t> {
        size_t m = i / 2;
        int64_t other = (i % 2 == 0) ? (int64_t)m - 1 : (int64_t)m + 1;
        return {m, (size_t)std::clamp<int64_t>(other, 0, (int64_t)n - 1)};
    };
    auto [x0, x1] = taps(x, cw);
    auto [y0, y1] = taps(y, ch);
    auto row = [&](size_t yy) { return coarse[yy * cw + x0] * T(0.75) + coarse[yy * cw + x1] * T(0.25); };
    return row(y0) * T(0.75) + row(y1) * T(0.25);
}
template <class T> void bloom_apply(std::vector<V3<T>>& hdr, size_t width, size_t height) {  // bloom.rs:93-125
    if (width == 0 || height == 0) return;
    std::vector<V3<T>> pyr(pyramid_len(width, height));
    std::copy(hdr.begin(), hdr.begin() + width * height, pyr.begin());
    for (size_t k = 1; k <= BLOOM_LEVELS; ++k) bloom_downsample(pyr, width, height, k);
    for (size_t k = BLOOM_LEVELS - 1; k >= 1; --k) {
        auto [w, h] = level_size(width, height, k);
        auto [cw, ch] = level_size(width, height, k + 1);
        size_t off = level_offset(width, height, k);
        const V3<T>* coarse = &pyr[off + w * h];
        for (size_t y = 0; y < h; ++y)
            for (size_t x = 0; x < w; ++x) pyr[off + y * w + x] += upsample_at(coarse, cw, ch, x, y);
    }
    auto [w1, h1] = level_size(width, height, 1);
    const V3<T>* lvl1 = &pyr[level_offset(width, height, 1)];
    T halo = T(BLOOM_STRENGTH) / T(BLOOM_LEVELS);
    for (size_t y = 0; y < height; ++y)
        for (size_t x = 0; x < width; ++x) {
            V3<T>& px = hdr[y * width + x];
            px = px * (T(1) - T(BLOOM_STRENGTH)) + upsample_at(lvl1, w1, h1, x, y) * halo;
        }
}

// ------------------------------------------------------------------------------------------
// Gamma LUT and pack (renderer.rs:1102-1134), glyphs (hud.rs:473-532).
// ------------------------------------------------------------------------------------------
constexpr size_t GAMMA_LUT_SIZE = 4096;
inline const std::array<uint8_t, GAMMA_LUT_SIZE>& gamma_lut() {
    static std::array<uint8_t, GAMMA_LUT_SIZE> lut = [] {
        std::array<uint8_t, GAMMA_LUT_SIZE> t{};
        for (size_t i = 0; i < GAMMA_LUT_SIZE; ++i) {
            float x = (float)i / (float)(GAMMA_LUT_SIZE - 1);
            float v = clamp_(::powf(x, 1.0f / 2.2f) * 255.0f + 0.5f, 0.0f, 255.0f);
            t[i] = (uint8_t)v;
        }
        return t;
    }();
    return lut;
}
template <class T> inline uint32_t pack_rgb(const V3<T>& c) {
    const auto& lut = gamma_lut();
    V3<T> mapped = V3<T>(c.x / (T(1) + c.x * T(0.35)), c.y / (T(1) + c.y * T(0.35)), c.z / (T(1) + c.z * T(0.35)))
                       .clamp(T(0), T(1));
    T scale = T(GAMMA_LUT_SIZE - 1);
    uint32_t r = lut[as_usize(mapped.x * scale)], g = lut[as_usize(mapped.y * scale)],
             b = lut[as_usize(mapped.z * scale)];
    return (r << 16) | (g << 8) | b;
}
inline std::array<uint8_t, 7> glyph_5x7(char ch) {
    switch (ch) {
        case '0': return {0b01110, 0b10001, 0b10011, 0b10101, 0b11001, 0b10001, 0b01110};
        case '1': return {0b00100, 0b01100, 0b00100, 0b00100, 0b00100, 0b00100, 0b01110};
        case '2': return {0b01110, 0b10001, 0b00001, 0b00010, 0b00100, 0b01000, 0b11111};
        case '3': return {0b11110, 0b00001, 0b00001, 0b01110, 0b00001, 0b00001, 0b11110};
        case '4': return {0b00010, 0b00110, 0b01010, 0b10010, 0b11111, 0b00010, 0b00010};
        case '5': return {0b11111, 0b10000, 0b11110, 0b00001, 0b00001, 0b10001, 0b01110};
        case '6': return {0b01110, 0b10000, 0b10000, 0b11110, 0b10001, 0b10001, 0b01110};
        case '7': return {0b11111, 0b00001, 0b00010, 0b00100, 0b01000, 0b01000, 0b01000};
        case '8': return {0b01110, 0b10001, 0b10001, 0b01110, 0b10001, 0b10001, 0b01110};
        case '9': return {0b01110, 0b10001, 0b10001, 0b01111, 0b00001, 0b00001, 0b01110};
        case '.': return {0b00000, 0b00000, 0b00000, 0b00000, 0b00000, 0b01100, 0b01100};
        case '-': return {0b00000, 0b00000, 0b00000, 0b11111, 0b00000, 0b00000, 0b00000};
        case '+': return {0b00000, 0b00100, 0b00100, 0b11111, 0b00100, 0b00100, 0b00000};
        case 'S': return {0b01111, 0b10000, 0b10000, 0b01110, 0b00001, 0b00001, 0b11110};
        default: return {0, 0, 0, 0, 0, 0, 0};
    }
}

// ------------------------------------------------------------------------------------------
// Renderer types (renderer.rs:10-312).
// ------------------------------------------------------------------------------------------
enum RenderMode : uint32_t { SHADED = 0, ISOCHRONES = 1, INSPECTOR = 2, DECISION_AGE = 3 };
enum ViewMode : uint32_t { PAST_LIGHT_CONE = 0, CAMERA_SIMULTANEITY = 1, FRONTIER = 2, PROPHECY = 3 };
enum ShadowMode : uint32_t { SHADOW_OFF = 0, LORENTZ_INVARIANT = 1, CAMERA_SLICE = 2 };
constexpr float FRONTIER_RAY_OFFSET = 0.14f;
constexpr size_t MAX_FLASHES = 16;
constexpr size_t MAX_REMOTE_FRONTIERS = 4;

template <class T> struct Camera4D {
    V4<T> position;
    Tetrad<T> tetrad = Tetrad<T>::rest();
    T proper_time = 0;
    T fov_y_rad = 0;
};
struct RenderConfig {
    size_t width = 0, height = 0;
    RenderMode mode = SHADED;
    ShadowMode shadow_mode = SHADOW_OFF;
    ViewMode slice_mode = PAST_LIGHT_CONE;
    float prophecy_delta = 3.5f;
    // Row sampling for the timed CPU baseline: when full_height > 0 the frame has full_height
    // rows and output row k is frame row row_offset + k * row_stride (height rows in all).
    size_t full_height = 0, row_stride = 1, row_offset = 0;
    size_t frame_height() const { return full_height ? full_height : height; }
    size_t frame_row(size_t k) const { return full_height ? row_offset + k * row_stride : k; }
};
template <class T> struct FlashEvent { V4<T> at; T width, intensity; V3<T> color; };
template <class T> struct Frontier { V4<T> origin; T proper_time; };
template <class T> struct FrameDynamics {
    bool has_frontier = false;
    Frontier<T> frontier;
    std::vector<FlashEvent<T>> flashes;
    T frontier_lag = 0;
    std::vector<V4<T>> remote_origins;
    T frontier_view_offset() const { return T(FRONTIER_RAY_OFFSET) + frontier_lag; }
    size_t n_flashes() const { return std::min(flashes.size(), MAX_FLASHES); }
    Frontier<T> frontier_or_camera(const Camera4D<T>& cam) const {
        return has_frontier ? frontier : Frontier<T>{cam.position, cam.proper_time};
    }
    std::vector<V4<T>> haze_origins(const Camera4D<T>& cam, ViewMode sm) const {
        std::vector<V4<T>> out;
        size_t nr = std::min(remote_origins.size(), MAX_REMOTE_FRONTIERS);
        if (sm == PROPHECY) {
            out.push_back(frontier_or_camera(cam).origin);
            for (size_t i = 0; i < nr; ++i) out.push_back(remote_origins[i]);
        } else if (sm == CAMERA_SIMULTANEITY) {
            for (size_t i = 0; i < nr; ++i) out.push_back(remote_origins[i]);
        }
        return out;
    }
};

template <class T> struct Scene {
    Bvh<T> bvh;
    std::vector<Material<T>> materials;
    V3<T> light_pos;
    std::vector<PointStar<T>> stars;
    std::vector<T> star_cn;  // color_norm per star
    void finish_stars() {
        star_cn.clear();
        for (auto& s : stars) star_cn.push_back(color_norm(s));
    }
};

template <class T> inline T analytic_decision_age(const V4<T>& event, const V4<T>& origin, const V4<T>& u) {
    V4<T> d = event - origin;
    T time_ago = d.mdot(u);
    T dist = m_sqrt(fmax_(time_ago * time_ago + d.mnorm_sq(), T(0)));
    return time_ago + dist;
}

template <class T> V3<T> hsv_to_rgb(T h_deg, T s, T v) {  // renderer.rs:1081-1100
    T c = v * s;
    T h = rem_euclid(h_deg / T(60), T(6));
    T x = c * (T(1) - std::fabs(rem_euclid(h, T(2)) - T(1)));
    T m = v - c;
    T r, g, b;
    if (h < T(1)) { r = c; g = x; b = 0; }
    else if (h < T(2)) { r = x; g = c; b = 0; }
    else if (h < T(3)) { r = 0; g = c; b = x; }
    else if (h < T(4)) { r = 0; g = x; b = c; }
    else if (h < T(5)) { r = x; g = 0; b = c; }
    else { r = c; g = 0; b = x; }
    return V3<T>(r + m, g + m, b + m);
}
template <class T> V3<T> decision_age_color(T age) {  // renderer.rs:494-507
    if (age < T(0)) return V3<T>(T(0.14), T(0.14), T(0.18));
    V3<T> col = hsv_to_rgb(fmin_(age * T(4), T(240)), T(0.82), T(0.88));
    if (age < T(0.45)) {
        T f = T(1) - age / T(0.45);
        col = col * (T(1) - f * T(0.7)) + V3<T>(T(1), T(0.96), T(0.65)) * (f * T(0.9));
    }
    if (std::fabs(rem_euclid(age * T(0.5), T(1)) - T(0.5)) > T(0.465)) col = V3<T>(T(0.95), T(0.98), T(1));
    return col;
}
template <class T> V3<T> apply_undecided_haze(const V3<T>& base, const V4<T>& event, const std::vector<V4<T>>& origins) {
    const T SHELL = T(0.18);  // renderer.rs:514-541
    T inside = -std::numeric_limits<T>::infinity();
    for (auto& o : origins) {
        V4<T> d = event - o;
        inside = fmax_(inside, d.t - d.spatial().length());
    }
    if (inside <= -SHELL) return base;
    V3<T> col = base;
    if (std::fabs(inside) < SHELL) {
        T k = T(1) - std::fabs(inside) / SHELL;
        col += V3<T>(T(0.45), T(0.92), T(1)) * (T(0.85) * k * k);
    }
    if (inside > T(0)) {
        T ripple = T(0.5) + T(0.5) * m_sin(event.x * T(3.5) + event.z * T(3.5) - event.t * T(4)) * m_cos(inside * T(5));
        const V3<T> HAZE(T(0.32), T(0.18), T(0.62));
        V3<T> haze = HAZE * (T(1) - T(0.35) * ripple) + V3<T>(T(0.18), T(0.72), T(0.92)) * (T(0.35) * ripple);
        T alpha = T(0.55) + T(0.25) * fmin_(inside * T(0.5), T(1));
        col = col * (T(1) - alpha) + haze * alpha;
    }
    return col;
}

template <class T> T clock_tile_central_proper_time(T u_tile, T v_tile, T grid_scale, T local_tau, T gu, T gv) {
    T inv_grid = T(1) / fmax_(grid_scale, T(1e-4));  // renderer.rs:704-715
    T delta_u = (u_tile - T(0.5)) * inv_grid;
    T delta_v = (v_tile - T(0.5)) * inv_grid;
    return local_tau - (delta_u * gu + delta_v * gv);
}
template <class T> bool point_on_hand(T dx, T dy, T angle_cw, T length, T half_width, T back) {
    T hx = m_sin(angle_cw), hy = m_cos(angle_cw);  // renderer.rs:930-943
    T proj_along = dx * hx + dy * hy;
    T proj_perp = std::fabs(dx * hy - dy * hx);
    return proj_along >= -back && proj_along <= length && proj_perp <= half_width;
}
template <class T> bool sample_digital_tau(T u, T v, T proper_time) {  // renderer.rs:946-981
    T rel_u = (u - T(0.28)) / (T(0.72) - T(0.28));
    T rel_v = (T(0.18) - v) / (T(0.18) - T(0.06));
    const uint64_t total_cols = 35;
    uint64_t col = as_usize(std::floor(rel_u * (T)total_cols));
    uint64_t row = as_usize(std::floor(rel_v * T(7)));
    if (col >= total_cols || row >= 7) return false;
    uint64_t char_idx = col / 6, char_col = col % 6;
    if (char_idx >= 6 || char_col >= 5) return false;
    int32_t t_tenths = as_i32(round_(proper_time * T(10)));
    char sign_ch = t_tenths < 0 ? '-' : '+';
    uint32_t abs_t = t_tenths < 0 ? (uint32_t)(-(int64_t)t_tenths) : (uint32_t)t_tenths;
    uint32_t tenths = abs_t % 10, ones = (abs_t / 10) % 10, tens = (abs_t / 100) % 10;
    char ch;
    switch (char_idx) {
        case 0: ch = sign_ch; break;
        case 1: ch = (char)('0' + tens); break;
        case 2: ch = (char)('0' + ones); break;
        case 3: ch = '.'; break;
        case 4: ch = (char)('0' + tenths); break;
        default: ch = 'S';
    }
    return ((glyph_5x7(ch)[row] >> (4 - char_col)) & 1) != 0;
}
template <class T> V3<T> sample_corner_mini_clock(T mdx, T mdy, T mr, T mini_tau, const Material<T>& mat) {
    if (mr > T(0.080)) return mat.base_color * T(1.15);  // renderer.rs:880-927
    const T TAU = C<T>::TAU;
    T angle = rem_euclid(m_atan2(mdx, mdy), TAU);
    T fast_angle = rem_euclid((mini_tau / T(1)) * TAU, TAU);
    T main_angle = rem_euclid((mini_tau / T(10)) * TAU, TAU);
    V3<T> col(T(0.04), T(0.06), T(0.10));
    if (angle <= fast_angle && mr < T(0.066)) col += mat.base_color * T(0.25);
    if (mr >= T(0.062) && mr <= T(0.078)) {
        T sector = angle / (TAU / T(10));
        T dist_to_tick = std::fabs(sector - round_(sector));
        int32_t tick_idx = as_i32(round_(sector)) % 10;
        bool is_cardinal = tick_idx == 0 || tick_idx == 5;
        T half_w = is_cardinal ? T(0.13) : T(0.07);
        if (dist_to_tick < half_w) return tick_idx == 0 ? V3<T>(T(1), T(0.88), T(0.15)) : V3<T>(T(0.80), T(0.85), T(0.92));
    }
    if (point_on_hand(mdx, mdy, fast_angle, T(0.068), T(0.0065), T(0.008))) return V3<T>(T(0.25), T(0.98), T(1));
    if (point_on_hand(mdx, mdy, main_angle, T(0.052), T(0.0085), T(0.008))) return V3<T>(T(1), T(0.95), T(0.30));
    if (mr < T(0.012)) return V3<T>(T(1), T(1), T(1));
    return col;
}
template <class T> V3<T> sample_clock_face_texture(const HitRecord<T>& hit, const Material<T>& mat) {
    const T TAU = C<T>::TAU;  // renderer.rs:737-874
    T grid_scale = fmax_(mat.grid_scale, T(1e-4));
    T inv_grid = T(1) / grid_scale;
    T u = rem_euclid(hit.uv_u * grid_scale, T(1));
    T v = rem_euclid(hit.uv_v * grid_scale, T(1));
    T central = clock_tile_central_proper_time(u, v, grid_scale, hit.proper_time, hit.grad_u, hit.grad_v);
    const T CC[4][2] = {{T(0.135), T(0.865)}, {T(0.865), T(0.865)}, {T(0.135), T(0.135)}, {T(0.865), T(0.135)}};
    for (int i = 0; i < 4; ++i) {
        T mc_x = CC[i][0], mc_y = CC[i][1];
        T mdx = u - mc_x, mdy = v - mc_y;
        T mr = m_sqrt(mdx * mdx + mdy * mdy);
        if (mr <= T(0.095)) {
            T corner_osc_tau = central + ((mc_x - T(0.5)) * inv_grid) * hit.grad_u + ((mc_y - T(0.5)) * inv_grid) * hit.grad_v;
            T mdx_phys = (mdx * inv_grid) * hit.uvs_u;
            T mdy_phys = (mdy * inv_grid) * hit.uvs_v;
            T mr_phys = m_sqrt(mdx_phys * mdx_phys + mdy_phys * mdy_phys);
            return sample_corner_mini_clock(mdx, mdy, mr, corner_osc_tau - mr_phys, mat);
        }
    }
    if (v >= T(0.035) && v <= T(0.205) && u >= T(0.25) && u <= T(0.75)) {
        if (!(v >= T(0.050) && v <= T(0.190)) || !(u >= T(0.265) && u <= T(0.735))) return mat.base_color * T(0.9);
        if (v >= T(0.06) && v <= T(0.18) && u >= T(0.28) && u <= T(0.72) && sample_digital_tau(u, v, central))
            return V3<T>(T(1), T(0.96), T(0.30));
        return V3<T>(T(0.03), T(0.04), T(0.07));
    }
    T cx = T(0.50), cy = T(0.57);
    T dx = u - cx, dy = v - cy;
    T r = m_sqrt(dx * dx + dy * dy);
    if (r > T(0.330)) {
        int32_t gu = as_i32(std::floor(u * T(4))), gv = as_i32(std::floor(v * T(4)));
        return rem_euclid_i32(wrap_add(gu, gv), 2) == 0 ? mat.base_color * T(0.78) : mat.checker_color * T(0.78);
    }
    if (r > T(0.292)) return mat.base_color * T(1.15);
    T dx_phys = (dx * inv_grid) * hit.uvs_u;
    T dy_phys = (dy * inv_grid) * hit.uvs_v;
    T r_phys = m_sqrt(dx_phys * dx_phys + dy_phys * dy_phys);
    T dial_tau = central - r_phys;
    T angle = rem_euclid(m_atan2(dx, dy), TAU);
    T main_hand_angle = rem_euclid((dial_tau / T(10)) * TAU, TAU);
    V3<T> dial_col(T(0.04), T(0.06), T(0.10));
    if (angle <= main_hand_angle && r < T(0.236)) dial_col += mat.base_color * T(0.22);
    if (r >= T(0.220) && r <= T(0.286)) {
        T sector = angle / (TAU / T(10));
        T dist_to_tick = std::fabs(sector - round_(sector));
        int32_t tick_idx = as_i32(round_(sector)) % 10;
        bool is_cardinal = tick_idx == 0 || tick_idx == 5;
        T half_w = is_cardinal ? T(0.105) : T(0.055);
        T inner_r = is_cardinal ? T(0.218) : T(0.242);
        if (dist_to_tick < half_w && r >= inner_r) {
            if (tick_idx == 0) return V3<T>(T(1), T(0.88), T(0.15));
            if (is_cardinal) return V3<T>(T(1), T(1), T(1));
            return V3<T>(T(0.75), T(0.80), T(0.88));
        }
    }
    T fast_angle = rem_euclid((dial_tau / T(1)) * TAU, TAU);
    if (point_on_hand(dx, dy, fast_angle, T(0.254), T(0.012), T(0.025))) return V3<T>(T(0.25), T(0.98), T(1));
    if (point_on_hand(dx, dy, main_hand_angle, T(0.228), T(0.022), T(0.025))) return V3<T>(T(1), T(0.95), T(0.30));
    if (point_on_hand(dx, dy, main_hand_angle, T(0.236), T(0.030), T(0.025))) return V3<T>(T(0.02), T(0.02), T(0.04));
    T slow_angle = rem_euclid((dial_tau / T(100)) * TAU, TAU);
    if (point_on_hand(dx, dy, slow_angle, T(0.162), T(0.026), T(0.025))) return V3<T>(T(1), T(0.35), T(0.25));
    if (r < T(0.034)) return V3<T>(T(1), T(1), T(1));
    return dial_col;
}
template <class T> T light_clock_bounce_fraction(T proper_time, T cavity_length) {
    T period = fmax_(T(2) * cavity_length, T(1e-4));  // renderer.rs:988-996
    T cycle = rem_euclid(proper_time / period, T(1));
    return cycle < T(0.5) ? cycle * T(2) : (T(1) - cycle) * T(2);
}
template <class T> V3<T> sample_light_clock_texture(T uv_u, T uv_v, T proper_time, const Material<T>& mat) {
    T u = rem_euclid(uv_u * mat.grid_scale, T(1));  // renderer.rs:1003-1052
    T v = rem_euclid(uv_v * mat.grid_scale, T(1));
    if (!(u >= T(0.12) && u <= T(0.88))) return mat.base_color * T(0.65);
    if ((v >= T(0.04) && v <= T(0.10)) || (v >= T(0.90) && v <= T(0.96))) return V3<T>(T(0.75), T(0.90), T(0.98));
    if (!(v >= T(0.10) && v <= T(0.90))) return V3<T>(T(0.08), T(0.12), T(0.16));
    T bounce = light_clock_bounce_fraction(proper_time, mat.cavity_length);
    T photon_v = T(0.10) + T(0.80) * bounce;
    T dv = std::fabs(v - photon_v), du = std::fabs(u - T(0.5));
    T dist = m_sqrt(du * du * T(0.7) + dv * dv);
    V3<T> col(T(0.05), T(0.09), T(0.13));
    T ruler_tick = rem_euclid((v - T(0.10)) / T(0.80) * T(8), T(1));
    if ((u < T(0.22) || u > T(0.78)) && ruler_tick < T(0.08)) col += V3<T>(T(0.20), T(0.35), T(0.35));
    if (du < T(0.015)) col += V3<T>(T(0.06), T(0.16), T(0.16));
    if (dv < T(0.032)) {
        T k = T(1) - dv / T(0.032);
        col += mat.base_color * (T(0.9) * (k * k));
    }
    if (dist < T(0.11)) {
        T k = T(1) - dist / T(0.11);
        col += V3<T>(T(1), T(1), T(0.85)) * (T(1.4) * (k * k));
    }
    return col;
}
template <class T> V3<T> sample_surface_albedo(const HitRecord<T>& hit, const Material<T>& mat) {
    V3<T> albedo;  // renderer.rs:544-580
    if (mat.pattern == CHECKERBOARD) {
        int32_t gu = as_i32(std::floor(hit.uv_u * mat.grid_scale));
        int32_t gv = as_i32(std::floor(hit.uv_v * mat.grid_scale));
        V3<T> col = rem_euclid_i32(wrap_add(gu, gv), 2) == 0 ? mat.base_color : mat.checker_color;
        T min_tri = fmin_(fmin_(hit.tri_bary.x, hit.tri_bary.y), hit.tri_bary.z);
        if (min_tri < mat.wireframe_width) {
            T edge_t = clamp_(min_tri / mat.wireframe_width, T(0), T(1));
            col = V3<T>::splat(T(0.07)) * (T(1) - edge_t) + col * edge_t;
        }
        albedo = col;
    } else if (mat.pattern == CLOCK_FACE) {
        albedo = sample_clock_face_texture(hit, mat);
    } else {
        albedo = sample_light_clock_texture(hit.uv_u, hit.uv_v, hit.proper_time, mat);
    }
    if (mat.pattern != CHECKERBOARD) {
        T u_tile = rem_euclid(hit.uv_u * mat.grid_scale, T(1));
        T v_tile = rem_euclid(hit.uv_v * mat.grid_scale, T(1));
        T border = fmin_(fmin_(u_tile, T(1) - u_tile), fmin_(v_tile, T(1) - v_tile));
        if (border < T(0.025)) albedo = albedo * T(0.35);
    }
    return albedo;
}
template <class T> V3<T> shade_sky_gradient(const V4<T>& ray_dir) {  // renderer.rs:1056-1062
    V3<T> s = ray_dir.spatial().normalized();
    T horizon = clamp_(s.y * T(0.5) + T(0.5), T(0), T(1));
    V3<T> zen(T(0.04), T(0.06), T(0.13)), hor(T(0.12), T(0.16), T(0.25));
    return hor * (T(1) - horizon) + zen * horizon;
}
template <class T> V3<T> shade_sky(const V4<T>& ray_dir) {  // renderer.rs:1064-1079
    V3<T> s = ray_dir.spatial().normalized();
    V3<T> sky = shade_sky_gradient(ray_dir);
    T theta = m_acos(clamp_(s.y, T(-1), T(1)));
    T phi = m_atan2(s.z, s.x);
    T grid_u = rem_euclid(phi / C<T>::PI * T(12), T(1));
    T grid_v = rem_euclid(theta / C<T>::PI * T(6), T(1));
    if (grid_u < T(0.025) || grid_v < T(0.025)) sky += V3<T>(T(0.06), T(0.09), T(0.14));
    return sky;
}
template <class T> V3<T> apply_distance_fog(const V3<T>& c, const V4<T>& ray_dir, T lambda) {
    T fog = m_exp(T(-0.008) * lambda);  // renderer.rs:691-695
    return c * fog + shade_sky_gradient(ray_dir) * (T(1) - fog);
}

// Per-pixel side outputs the parity harness compares.
template <class T> struct PixelAux {
    int64_t slot = -1;  // leaf slot of the primary hit (-1: miss)
    T lambda = 0, tau = 0;
    T min_bary = 0;     // smallest tet barycentric of the hit
    T denom_rel = 0;    // |N . d| / (|N| |d|)
    uint8_t shadow_rays = 0;
    TraceStats stats;   // primary + shadow traversal work
};

template <class T> struct Renderer {
    const Scene<T>& scene;
    const Camera4D<T>& camera;
    const RenderConfig& cfg;
    const FrameDynamics<T>& dyn;

    // renderer.rs:585-606.
    std::pair<V4<T>, T> light_emission_event(const V4<T>& hit_event) const {
        V3<T> to_light = scene.light_pos - hit_event.spatial();
        T dist = fmax_(to_light.length(), T(1e-4));
        T t_emit = cfg.shadow_mode == CAMERA_SLICE ? hit_event.t + camera.tetrad.beta().dot(to_light)
                                                   : hit_event.t - dist;
        return {V4<T>::from_time_space(t_emit, scene.light_pos), dist};
    }
    // renderer.rs:609-653.
    T compute_illumination(const V4<T>& ray_dir, const HitRecord<T>& hit, const Material<T>& mat, PixelAux<T>* aux) const {
        auto [emit, dist] = light_emission_event(hit.event);
        V4<T> to_light = (emit - hit.event) * (T(1) / dist);
        T cos_light = fmax_(rest_frame_cos(to_light, hit.normal, hit.four_vel), T(0));
        T cos_view = fmax_(-rest_frame_cos(ray_dir, hit.normal, hit.four_vel), T(0));
        if (mat.pattern == CHECKERBOARD) {
            bool in_shadow = false;
            if (cos_light > T(0) && cfg.shadow_mode != SHADOW_OFF) {
                if (aux) aux->shadow_rays++;
                in_shadow = scene.bvh.is_occluded(hit.event, to_light, T(2e-3), dist - T(2e-3), aux ? &aux->stats : nullptr);
            }
            T sf = in_shadow ? T(0.32) : T(1);
            T atten = T(1) / (T(1) + T(0.006) * dist * dist);
            return mat.emission + T(0.30) * cos_view + T(0.80) * sf * cos_light * atten;
        }
        return T(0.72) + T(0.38) * cos_view + T(0.22) * cos_light;
    }
    // renderer.rs:658-688.
    V3<T> compute_flash_illumination(const HitRecord<T>& hit, PixelAux<T>* aux) const {
        V3<T> total;
        for (size_t i = 0; i < dyn.n_flashes(); ++i) {
            const auto& f = dyn.flashes[i];
            T dt = hit.event.t - f.at.t;
            if (dt <= T(0)) continue;
            T dist = fmax_((f.at.spatial() - hit.event.spatial()).length(), T(1e-4));
            T shell_err = std::fabs(dt - dist);
            T half_w = fmax_(T(0.5) * f.width, T(1e-3));
            if (shell_err >= half_w) continue;
            T k = T(1) - shell_err / half_w;
            T pulse = k * k;
            V4<T> to_flash = (f.at - hit.event) * (T(1) / dist);
            T cos_f = fmax_(rest_frame_cos(to_flash, hit.normal, hit.four_vel), T(0));
            bool in_shadow = false;
            if (cos_f > T(0) && cfg.shadow_mode != SHADOW_OFF) {
                if (aux) aux->shadow_rays++;
                in_shadow = scene.bvh.is_occluded(hit.event, to_flash, T(2e-3), dist - T(2e-3), aux ? &aux->stats : nullptr);
            }
            T sf = in_shadow ? T(0.25) : T(1);
            T atten = T(1) / (T(1) + T(0.015) * dist * dist);
            total += f.color * (f.intensity * pulse * atten * (T(0.25) + T(0.75) * sf * cos_f));
        }
        return total;
    }
    // renderer.rs:414-489.
    V3<T> shade_hit(const V4<T>& ray_dir, const HitRecord<T>& hit, PixelAux<T>* aux) const {
        const Material<T>& mat = scene.materials[hit.material_id];
        switch (cfg.mode) {
            case SHADED: {
                V3<T> albedo = sample_surface_albedo(hit, mat);
                T lighting = compute_illumination(ray_dir, hit, mat, aux);
                V3<T> lit = albedo * lighting;
                if (dyn.n_flashes() > 0) {
                    V3<T> fr = compute_flash_illumination(hit, aux);
                    lit += (albedo * T(0.65) + V3<T>::splat(T(0.35))) * fr;
                }
                return apply_distance_fog(lit, ray_dir, hit.lambda);
            }
            case ISOCHRONES: {
                T phase = rem_euclid(hit.lambda * T(0.12), T(1));
                V3<T> base = hsv_to_rgb(phase * T(300), T(0.8), T(0.85));
                T t_contour = std::fabs(rem_euclid(hit.event.t, T(1)) - T(0.5));
                T tau_contour = std::fabs(rem_euclid(hit.proper_time, T(1)) - T(0.5));
                if (t_contour > T(0.45)) return V3<T>(T(1), T(1), T(1));
                if (tau_contour > T(0.46)) return V3<T>(T(0.1), T(0.1), T(0.1));
                return base;
            }
            case INSPECTOR: {
                const auto& b = hit.tet_bary;
                T min_b = fmin_(fmin_(fmin_(b[0], b[1]), b[2]), b[3]);
                T edge = min_b < T(0.035) ? T(0.12) : T(1);
                T speed = clamp_((hit.four_vel.t - T(1)) * T(0.8), T(0), T(1));
                V3<T> tint(T(0.25) + T(0.65) * b[1] + T(0.3) * speed, T(0.25) + T(0.65) * b[2],
                           T(0.35) + T(0.55) * b[3] * (T(1) - T(0.5) * speed));
                return tint * edge;
            }
            default: {
                Frontier<T> fr = dyn.frontier_or_camera(camera);
                T age = hit.decided_at > T(DECIDED_AT_STATIC) * T(0.5)
                            ? fr.proper_time - hit.decided_at
                            : analytic_decision_age(hit.event, fr.origin, camera.tetrad.e[0]);
                T cos_view = fmax_(-rest_frame_cos(ray_dir, hit.normal, hit.four_vel), T(0));
                return apply_distance_fog(decision_age_color(age) * (T(0.55) + T(0.45) * cos_view), ray_dir, hit.lambda);
            }
        }
    }

    // Per-frame constants of render_frame (renderer.rs:334-358).
    struct Frame {
        T half_h, half_w, pixel_pitch, cone;
        V4<T> ray_origin, e0;
        bool draw_stars;
        std::vector<V4<T>> haze;
    };
    Frame frame() const {
        Frame f;
        size_t w = cfg.width, h = cfg.frame_height();
        T aspect = (T)w / (T)h;
        f.half_h = m_tan(T(0.5) * camera.fov_y_rad);
        f.half_w = aspect * f.half_h;
        f.haze = dyn.haze_origins(camera, cfg.slice_mode);
        f.ray_origin = camera.position;
        if (cfg.slice_mode == FRONTIER) f.ray_origin = camera.position - camera.tetrad.e[0] * dyn.frontier_view_offset();
        else if (cfg.slice_mode == PROPHECY) f.ray_origin = camera.position + camera.tetrad.e[0] * T(cfg.prophecy_delta);
        f.cone = cfg.slice_mode == PAST_LIGHT_CONE ? T(-1) : cfg.slice_mode == FRONTIER ? T(1) : T(0);
        f.e0 = camera.tetrad.e[0];
        f.draw_stars = cfg.mode == SHADED && !scene.stars.empty();
        f.pixel_pitch = T(2) * f.half_h / (T)h;
        return f;
    }

    // The body of render_frame's pixel loop (renderer.rs:369-404): HDR radiance of pixel (px, py).
    V3<T> pixel(size_t px, size_t py, const Frame& fr, PixelAux<T>* aux) const {
        size_t w = cfg.width, h = cfg.frame_height();
        const T half_h = fr.half_h, half_w = fr.half_w, cone = fr.cone, pixel_pitch = fr.pixel_pitch;
        const V4<T>& ray_origin = fr.ray_origin;
        const V4<T>& e0 = fr.e0;
        const bool draw_stars = fr.draw_stars;
        const std::vector<V4<T>>& haze = fr.haze;

        T ndc_y = T(1) - T(2) * (((T)py + T(0.5)) / (T)h);
        T sy = ndc_y * half_h;
        T ndc_x = T(2) * (((T)px + T(0.5)) / (T)w) - T(1);
        T sx = ndc_x * half_w;
        V3<T> local_dir = V3<T>(sx, sy, T(1)).normalized();
        V4<T> ray_dir;
        if (cfg.slice_mode == PAST_LIGHT_CONE) ray_dir = camera.tetrad.past_light_ray_direction(local_dir);
        else if (cfg.slice_mode == FRONTIER) ray_dir = camera.tetrad.future_light_ray_direction(local_dir);
        else ray_dir = camera.tetrad.local_spatial_to_world(local_dir);

        HitRecord<T> hit;
        int64_t slot = -1;
        bool found = scene.bvh.trace(ray_origin, ray_dir, T(1e-3), T(180), &hit, &slot, aux ? &aux->stats : nullptr);
        V3<T> color;
        if (found) {
            if (aux) {
                aux->slot = slot;
                aux->lambda = hit.lambda;
                aux->tau = hit.proper_time;
                aux->min_bary = fmin_(fmin_(fmin_(hit.tet_bary[0], hit.tet_bary[1]), hit.tet_bary[2]), hit.tet_bary[3]);
                const Geom<T>& g = scene.bvh.hot[(size_t)slot];
                aux->denom_rel = std::fabs(g.n.edot(ray_dir)) / (g.n.elen() * ray_dir.elen());
            }
            V3<T> shaded = shade_hit(ray_dir, hit, aux);
            color = haze.empty() ? shaded : apply_undecided_haze(shaded, hit.event, haze);
        } else {
            color = shade_sky(ray_dir);
        }
        if (draw_stars) {
            T inv_len = T(1) / m_sqrt(sx * sx + sy * sy + T(1));
            T spread = pixel_pitch * inv_len * m_sqrt(inv_len);
            T lambda_max = found ? hit.lambda : std::numeric_limits<T>::infinity();
            color += star_light(scene.stars, scene.star_cn, ray_origin, ray_dir, e0, cone, T(0), spread, lambda_max);
        }
        return color;
    }

    // renderer.rs:327-412 — rows spread over `threads` workers through a shared row counter
    // (rayon's par_chunks_mut), bloom serial, then the LUT pack. `hdr_out` (optional) receives
    // the pre-bloom radiance.
    void render(uint32_t* framebuffer, std::vector<PixelAux<T>>* aux, std::vector<V3<T>>* hdr_out,
                unsigned threads) const {
        size_t w = cfg.width, h = cfg.height;
        const Frame fr = frame();
        std::vector<V3<T>> hdr(w * h);
        if (aux) aux->assign(w * h, PixelAux<T>());
        std::atomic<size_t> next_row{0};
        auto work = [&] {
            for (;;) {
                size_t py = next_row.fetch_add(1);
                if (py >= h) break;
                for (size_t px = 0; px < w; ++px)
                    hdr[py * w + px] = pixel(px, cfg.frame_row(py), fr, aux ? &(*aux)[py * w + px] : nullptr);
            }
        };
        if (threads <= 1) work();
        else {
            std::vector<std::thread> pool;
            for (unsigned i = 0; i < threads; ++i) pool.emplace_back(work);
            for (auto& t : pool) t.join();
        }
        if (hdr_out) *hdr_out = hdr;
        bloom_apply(hdr, w, h);
        for (size_t i = 0; i < w * h; ++i) framebuffer[i] = pack_rgb(hdr[i]);
    }
};

}  // namespace orc
