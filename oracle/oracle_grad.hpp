// TEST INFRASTRUCTURE ONLY — part of the CPU oracle that the parity tests use as the checker.
// Nothing in the shipped library includes, links or calls this file.
//
// The image loss of a frame with its discrete outcomes frozen, in the oracle's scalar type: the
// FP64 reference for the engine's gradient (sr_adjoint). `freeze` renders the frame at theta0 and
// records per pixel the hit tetrahedron and hit record, the surface albedo, the main light's shadow
// test, the sky's grid line and the stars whose footprint passed the cut. `frozen_hdr` then
// evaluates the HDR image at another observer with those outcomes held fixed: the camera ray, the
// hit parameter on the same tetrahedron's hyperplane, the light's emission event, the rest-frame
// cosines, attenuation and fog, the sky gradient, and every passed star's cone crossing (on the
// segment the search finds at theta), footprint kernel, Doppler factor and blackbody colour. The
// loss compares `level` 2x2-box halvings of that image with the target's. Covered frames: shaded
// mode, past light cone, no flashes, no haze. Central differences of this smooth function give
// the FP64 reference gradient.
//
// Reference: the per-pixel path of render_frame (renderer.rs:342-404), compute_illumination
// (renderer.rs:609-653), star_light (star.rs:240-286), as restated in oracle_render.hpp.
#pragma once
#include <atomic>
#include <thread>

#include "oracle_render.hpp"

namespace orc {

template <class T> struct FrozenPixel {
    int64_t slot = -1;
    HitRecord<T> hit{};
    V3<T> albedo;
    bool shadow = false;
    bool grid = false;
    std::vector<uint32_t> pass;
};

template <class T> struct FrozenFrame {
    size_t w = 0, h = 0;
    std::vector<FrozenPixel<T>> px;
};

// The camera ray of pixel (px, py) on the past light cone (Renderer::pixel's first lines).
template <class T>
inline void past_cone_ray(const Renderer<T>& R, const typename Renderer<T>::Frame& fr, size_t px, size_t py, V4<T>* o,
                          V4<T>* d, T* sx_out, T* sy_out) {
    size_t w = R.cfg.width, h = R.cfg.frame_height();
    T ndc_y = T(1) - T(2) * (((T)py + T(0.5)) / (T)h);
    T sy = ndc_y * fr.half_h;
    T ndc_x = T(2) * (((T)px + T(0.5)) / (T)w) - T(1);
    T sx = ndc_x * fr.half_w;
    V3<T> local_dir = V3<T>(sx, sy, T(1)).normalized();
    *d = R.camera.tetrad.past_light_ray_direction(local_dir);
    *o = fr.ray_origin;
    *sx_out = sx;
    *sy_out = sy;
}

// worldline_cone_event without its segment-range test: the crossing on the segment the search
// finds (the crossing moves continuously with the observer).
template <class T>
inline bool cone_crossing(const PointStar<T>& star, const V4<T>& origin, const V4<T>& e0, T cone, V4<T>* d_out,
                          V4<T>* u_out) {
    const auto& segs = star.segments;
    size_t lo = 0, hi = segs.size();
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (past_the_cone(segs[mid].event, origin, e0, cone) <= T(0)) lo = mid + 1;
        else hi = mid;
    }
    size_t idx = std::max<size_t>(lo, 1) - 1;
    if (idx >= segs.size()) return false;
    const auto& seg = segs[idx];
    T s = segment_cone_crossing(seg, origin, e0, cone);
    *d_out = seg.event - origin + seg.four_velocity * s;
    *u_out = seg.four_velocity;
    return true;
}

template <class T> inline bool sky_grid(const V4<T>& d) {
    V3<T> a = shade_sky(d), b = shade_sky_gradient(d);
    return !(a.x == b.x && a.y == b.y && a.z == b.z);
}

// `binning`: -1 bins the stars per pixel on star sets above 4096, 0 never, 1 always (the tests
// check that both give the same outcomes).
template <class T> FrozenFrame<T> freeze(const Renderer<T>& R, unsigned threads, int binning = -1) {
    FrozenFrame<T> F;
    F.w = R.cfg.width;
    F.h = R.cfg.height;
    F.px.resize(F.w * F.h);
    const auto fr = R.frame();
    const auto& stars = R.scene.stars;
    std::vector<char> ok(stars.size());
    std::vector<V4<T>> sd(stars.size()), su(stars.size());
    for (size_t i = 0; i < stars.size(); ++i) ok[i] = worldline_cone_event(stars[i], fr.ray_origin, fr.e0, fr.cone, &sd[i], &su[i]);
    // Candidate stars per pixel, in increasing star order. A star passes a pixel's footprint cut
    // only when the angle theta between its direction and the pixel's ray has tan(theta) < 2.4 *
    // spread <= 2.4 * pixel pitch * c^1.5 (c: cosine of the pixel's view angle). On the image
    // plane, where the pixel pitch is one pixel, that angle spans at most 2.4 / sqrt(c) pixels
    // (radial magnification 1 / c^2), so a star is listed at the pixels within a radius of
    // 1.25 * 2.4 / sqrt(c_min) + 2 pixels of where its direction projects; the exact test below
    // decides, as in the full loop over all stars, which it replaces on large star sets.
    std::vector<std::vector<uint32_t>> cand;
    const bool binned = fr.draw_stars && (binning > 0 || (binning < 0 && stars.size() > 4096));
    if (binned) {
        cand.resize(F.w * F.h);
        const double hw = (double)fr.half_w, hh = (double)fr.half_h;
        const double c_min = 1.0 / std::sqrt(1.0 + hw * hw + hh * hh);
        const int rad = (int)std::ceil(1.25 * 2.4 / std::sqrt(c_min)) + 2;
        const Tetrad<T>& tet = R.camera.tetrad;
        for (size_t i = 0; i < stars.size(); ++i) {
            if (!ok[i]) continue;
            T tau = -sd[i].mdot(fr.e0);
            V4<T> r = sd[i] + fr.e0 * (-tau);
            double x = (double)r.mdot(tet.e[1]), y = (double)r.mdot(tet.e[2]), z = (double)r.mdot(tet.e[3]);
            double len = std::sqrt(x * x + y * y + z * z);
            if (!(z > 0.25 * len)) continue;  // beyond 75 degrees of the axis: outside every view cone here
            double px = (x / z / hw + 1.0) * 0.5 * (double)F.w - 0.5, py = (1.0 - y / z / hh) * 0.5 * (double)F.h - 0.5;
            long x0 = std::max<long>(0, (long)std::floor(px) - rad), x1 = std::min<long>((long)F.w - 1, (long)std::ceil(px) + rad);
            long y0 = std::max<long>(0, (long)std::floor(py) - rad), y1 = std::min<long>((long)F.h - 1, (long)std::ceil(py) + rad);
            for (long yy = y0; yy <= y1; ++yy)
                for (long xx = x0; xx <= x1; ++xx) cand[(size_t)yy * F.w + (size_t)xx].push_back((uint32_t)i);
        }
    }
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (;;) {
            size_t py = next.fetch_add(1);
            if (py >= F.h) break;
            for (size_t px = 0; px < F.w; ++px) {
                FrozenPixel<T>& P = F.px[py * F.w + px];
                V4<T> o, d;
                T sx, sy;
                past_cone_ray(R, fr, px, py, &o, &d, &sx, &sy);
                int64_t slot = -1;
                HitRecord<T> hit{};
                bool found = R.scene.bvh.trace(o, d, T(1e-3), T(180), &hit, &slot, nullptr);
                T lambda_max = std::numeric_limits<T>::infinity();
                if (found) {
                    P.slot = slot;
                    P.hit = hit;
                    const Material<T>& mat = R.scene.materials[hit.material_id];
                    P.albedo = sample_surface_albedo(hit, mat);
                    auto [emit, dist] = R.light_emission_event(hit.event);
                    V4<T> to_light = (emit - hit.event) * (T(1) / dist);
                    T cos_light = fmax_(rest_frame_cos(to_light, hit.normal, hit.four_vel), T(0));
                    if (mat.pattern == CHECKERBOARD && cos_light > T(0) && R.cfg.shadow_mode != SHADOW_OFF)
                        P.shadow = R.scene.bvh.is_occluded(hit.event, to_light, T(2e-3), dist - T(2e-3), nullptr);
                    lambda_max = hit.lambda;
                } else {
                    P.grid = sky_grid(d);
                }
                if (!fr.draw_stars) continue;
                T inv_len = T(1) / m_sqrt(sx * sx + sy * sy + T(1));
                T spread = fr.pixel_pitch * inv_len * m_sqrt(inv_len);
                V4<T> n = d - fr.e0 * fr.cone;
                const std::vector<uint32_t>* list = binned ? &cand[py * F.w + px] : nullptr;
                const size_t m = binned ? list->size() : stars.size();
                for (size_t j = 0; j < m; ++j) {
                    const size_t i = binned ? (*list)[j] : j;
                    if (!ok[i]) continue;
                    T tau = -sd[i].mdot(fr.e0);
                    V4<T> r = sd[i] + fr.e0 * (-tau);
                    T along = r.mdot(n);
                    if (along <= T(0) || along >= lambda_max) continue;
                    V4<T> perp = r - n * along;
                    T d2 = fmax_(perp.mnorm_sq(), T(0));
                    T sigma = T(KERNEL_SIGMA) * (T(0) + spread * along);
                    T cut = T(KERNEL_CUTOFF_SIGMAS) * sigma;
                    if (d2 >= cut * cut) continue;
                    P.pass.push_back((uint32_t)i);
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < std::max(1u, threads); ++i) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    return F;
}

// The HDR image (w*h) at the renderer's observer under the frozen outcomes.
template <class T> std::vector<V3<T>> frozen_hdr(const Renderer<T>& R, const FrozenFrame<T>& F, unsigned threads) {
    std::vector<V3<T>> out(F.w * F.h);
    const auto fr = R.frame();
    const auto& stars = R.scene.stars;
    std::vector<char> ok(stars.size());
    std::vector<V4<T>> sd(stars.size()), su(stars.size());
    for (size_t i = 0; i < stars.size(); ++i) ok[i] = cone_crossing(stars[i], fr.ray_origin, fr.e0, fr.cone, &sd[i], &su[i]);
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (;;) {
            size_t py = next.fetch_add(1);
            if (py >= F.h) break;
            for (size_t px = 0; px < F.w; ++px) {
                const FrozenPixel<T>& P = F.px[py * F.w + px];
                V4<T> o, d;
                T sx, sy;
                past_cone_ray(R, fr, px, py, &o, &d, &sx, &sy);
                V3<T> color;
                if (P.slot >= 0) {
                    const Geom<T>& g = R.scene.bvh.hot[(size_t)P.slot];
                    T lambda = g.n.edot(g.v0 - o) / g.n.edot(d);
                    V4<T> ev = o + d * lambda;
                    auto [emit, dist] = R.light_emission_event(ev);
                    V4<T> to_light = (emit - ev) * (T(1) / dist);
                    T cos_light = fmax_(rest_frame_cos(to_light, P.hit.normal, P.hit.four_vel), T(0));
                    T cos_view = fmax_(-rest_frame_cos(d, P.hit.normal, P.hit.four_vel), T(0));
                    const Material<T>& mat = R.scene.materials[P.hit.material_id];
                    T lighting;
                    if (mat.pattern == CHECKERBOARD) {
                        bool in_shadow = P.shadow && cos_light > T(0) && R.cfg.shadow_mode != SHADOW_OFF;
                        T sf = in_shadow ? T(0.32) : T(1);
                        T atten = T(1) / (T(1) + T(0.006) * dist * dist);
                        lighting = mat.emission + T(0.30) * cos_view + T(0.80) * sf * cos_light * atten;
                    } else {
                        lighting = T(0.72) + T(0.38) * cos_view + T(0.22) * cos_light;
                    }
                    color = apply_distance_fog(P.albedo * lighting, d, lambda);
                } else {
                    color = shade_sky_gradient(d);
                    if (P.grid) color += V3<T>(T(0.06), T(0.09), T(0.14));
                }
                if (fr.draw_stars && !P.pass.empty()) {
                    T inv_len = T(1) / m_sqrt(sx * sx + sy * sy + T(1));
                    T spread = fr.pixel_pitch * inv_len * m_sqrt(inv_len);
                    V4<T> n = d - fr.e0 * fr.cone;
                    V3<T> total;
                    for (uint32_t i : P.pass) {
                        if (!ok[i]) continue;
                        T tau = -sd[i].mdot(fr.e0);
                        V4<T> r = sd[i] + fr.e0 * (-tau);
                        T along = r.mdot(n);
                        V4<T> perp = r - n * along;
                        T d2 = fmax_(perp.mnorm_sq(), T(0));
                        T sigma = T(KERNEL_SIGMA) * (T(0) + spread * along);
                        T inv_2s2 = T(1) / (T(2) * sigma * sigma);
                        T kernel = m_exp(-d2 * inv_2s2) * inv_2s2 * C<T>::FRAC_1_PI;
                        T doppler = T(1);
                        T lam = m_sqrt(fmax_(r.mnorm_sq(), T(0)));
                        T du = sd[i].mdot(su[i]);
                        if (du > T(0)) doppler = lam / du;
                        total += blackbody_rgb(stars[i].temperature * doppler) * (R.scene.star_cn[i] * kernel);
                    }
                    color += total;
                }
                out[py * F.w + px] = color;
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < std::max(1u, threads); ++i) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    return out;
}

// One 2x2-box halving with clamped taps (the loss's pyramid).
template <class T> std::vector<V3<T>> box_halve(const std::vector<V3<T>>& src, size_t sw, size_t sh, size_t* dw, size_t* dh) {
    *dw = (sw + 1) / 2;
    *dh = (sh + 1) / 2;
    std::vector<V3<T>> dst(*dw * *dh);
    for (size_t y = 0; y < *dh; ++y)
        for (size_t x = 0; x < *dw; ++x) {
            size_t x0 = 2 * x, x1 = std::min(2 * x + 1, sw - 1), y0 = 2 * y, y1 = std::min(2 * y + 1, sh - 1);
            const V3<T>&a = src[y0 * sw + x0], &b = src[y0 * sw + x1], &c = src[y1 * sw + x0], &e = src[y1 * sw + x1];
            dst[y * *dw + x] = V3<T>(((a.x + b.x) + (c.x + e.x)) * T(0.25), ((a.y + b.y) + (c.y + e.y)) * T(0.25),
                                     ((a.z + b.z) + (c.z + e.z)) * T(0.25));
        }
    return dst;
}

template <class T>
double pyramid_loss(std::vector<V3<T>> img, std::vector<V3<T>> tgt, size_t w, size_t h, unsigned level) {
    for (unsigned k = 0; k < level; ++k) {
        size_t nw, nh;
        img = box_halve(img, w, h, &nw, &nh);
        tgt = box_halve(tgt, w, h, &nw, &nh);
        w = nw;
        h = nh;
    }
    double L = 0.0;
    for (size_t i = 0; i < w * h; ++i) {
        double r[3] = {(double)img[i].x - (double)tgt[i].x, (double)img[i].y - (double)tgt[i].y,
                       (double)img[i].z - (double)tgt[i].z};
        L += r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    }
    return L;
}

}  // namespace orc
