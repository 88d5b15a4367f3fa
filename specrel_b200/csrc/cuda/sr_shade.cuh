// shade_hit and the per-pixel tail of render_frame (renderer.rs:369-404, 414-489, 609-688), generic
// over the any-hit query the shadow rays use (`Occ` is a callable (origin, dir, t_min, t_max) -> bool).
#pragma once
#include "sr_device.cuh"
#include "sr_kernels.h"

namespace srd {

// compute_illumination (renderer.rs:609-653).
template <class Occ>
__device__ __forceinline__ float illumination(const SrGpuUniforms& U, const Cam& cam, float4 dir, const Hit& h,
                                              const Mat& m, Occ& occ, uint32_t* shadow_rays) {
    float4 to_light;
    float dist;
    light_ray(U, cam, h.event, &to_light, &dist);
    float cl = fmaxf(rest_frame_cos(to_light, h.normal, h.four_vel), 0.0f);
    float cv = fmaxf(-rest_frame_cos(dir, h.normal, h.four_vel), 0.0f);
    if (m.pattern == 0u) {
        bool in_shadow = false;
        if (cl > 0.0f && U.shadow_mode != 0u) {
            ++*shadow_rays;
            in_shadow = occ(h.event, to_light, 2e-3f, dist - 2e-3f);
        }
        float sf = in_shadow ? 0.32f : 1.0f;
        float atten = 1.0f / (1.0f + 0.006f * dist * dist);
        return m.emission + 0.30f * cv + 0.80f * sf * cl * atten;
    }
    return 0.72f + 0.38f * cv + 0.22f * cl;
}

// compute_flash_illumination with the uniform block's premultiplied colours (gpu.rs:160-167).
template <class Occ>
static __device__ __noinline__ F3 flash_illumination(const SrGpuUniforms& U, float4 event, float4 normal, float4 four_vel,
                                                     Occ& occ, uint32_t* shadow_rays) {
    F3 total{0.0f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < U.num_flashes; ++i) {
        float4 at = v4(U.flash_at[i][0], U.flash_at[i][1], U.flash_at[i][2], U.flash_at[i][3]);
        float dt = event.x - at.x;
        if (dt <= 0.0f) continue;
        float dist = fmaxf(len3(sub(spatial(at), spatial(event))), 1e-4f);
        float err = fabsf(dt - dist);
        float hw = fmaxf(0.5f * U.flash_col_width[i][3], 1e-3f);
        if (err >= hw) continue;
        float k = 1.0f - err / hw;
        float pulse = k * k;
        float4 tf = mul4(sub4(at, event), 1.0f / dist);
        float cf = fmaxf(rest_frame_cos(tf, normal, four_vel), 0.0f);
        bool in_shadow = false;
        if (cf > 0.0f && U.shadow_mode != 0u) {
            ++*shadow_rays;
            in_shadow = occ(event, tf, 2e-3f, dist - 2e-3f);
        }
        float sf = in_shadow ? 0.25f : 1.0f;
        float atten = 1.0f / (1.0f + 0.015f * dist * dist);
        F3 c{U.flash_col_width[i][0], U.flash_col_width[i][1], U.flash_col_width[i][2]};
        total = add(total, mul(c, pulse * atten * (0.25f + 0.75f * sf * cf)));
    }
    return total;
}

// shade_hit (renderer.rs:414-489).
template <class Occ>
__device__ __forceinline__ F3 shade_hit(const srk::SceneDev& s, const SrGpuUniforms& U, const Cam& cam, float4 dir,
                                        const Hit& h, Occ& occ, uint32_t* shadow_rays) {
    Mat m = load_mat(s.mats, h.material);
    if (U.mode == 0u) {
        F3 albedo = surface_albedo(h, m, s.tables);
        float lighting = illumination(U, cam, dir, h, m, occ, shadow_rays);
        F3 lit = mul(albedo, lighting);
        if (U.num_flashes > 0u) {
            F3 fr = flash_illumination(U, h.event, h.normal, h.four_vel, occ, shadow_rays);
            lit = add(lit, mulv(add(mul(albedo, 0.65f), F3{0.35f, 0.35f, 0.35f}), fr));
        }
        return apply_fog(lit, dir, h.lambda);
    }
    if (U.mode == 1u) {
        float phase = rem_e(h.lambda * 0.12f, 1.0f);
        F3 base = hsv_to_rgb(phase * 300.0f, 0.8f, 0.85f);
        float tc = fabsf(rem_e(h.event.x, 1.0f) - 0.5f);
        float uc = fabsf(rem_e(h.tau, 1.0f) - 0.5f);
        if (tc > 0.45f) return F3{1.0f, 1.0f, 1.0f};
        if (uc > 0.46f) return F3{0.1f, 0.1f, 0.1f};
        return base;
    }
    if (U.mode == 2u) {
        float mb = fminf(fminf(fminf(h.b0, h.b1), h.b2), h.b3);
        float edge = mb < 0.035f ? 0.12f : 1.0f;
        float sp = clampf_((h.four_vel.x - 1.0f) * 0.8f, 0.0f, 1.0f);
        F3 tint{0.25f + 0.65f * h.b1 + 0.3f * sp, 0.25f + 0.65f * h.b2, 0.35f + 0.55f * h.b3 * (1.0f - 0.5f * sp)};
        return mul(tint, edge);
    }
    float4 fo = cam.frontier;
    float age;
    if (h.decided_at > -1.0e9f * 0.5f) {
        age = U.frontier_tau - h.decided_at;
    } else {  // analytic_decision_age (renderer.rs:319-325)
        float4 d = sub4(h.event, fo);
        float ta = mdot(d, cam.e0);
        age = ta + sqrtf(fmaxf(ta * ta + mdot(d, d), 0.0f));
    }
    float cv = fmaxf(-rest_frame_cos(dir, h.normal, h.four_vel), 0.0f);
    return apply_fog(mul(decision_age_color(age), 0.55f + 0.45f * cv), dir, h.lambda);
}

// Camera ray of pixel (px, py) (renderer.rs:342-384): origin and direction, plus the image-plane
// point (sx, sy) the star footprint needs.
__device__ __forceinline__ void camera_ray(const SrGpuUniforms& U, const Cam& c, uint32_t px, uint32_t py, float4* o,
                                           float4* d, float* sx_out, float* sy_out) {
    float w = (float)U.size[0], h = (float)U.size[1];
    float ndc_y = 1.0f - 2.0f * (((float)py + 0.5f) / h);
    float ndc_x = 2.0f * (((float)px + 0.5f) / w) - 1.0f;
    float sx = ndc_x * U.half_wh[0];
    float sy = ndc_y * U.half_wh[1];
    F3 ld = normalized3(F3{sx, sy, 1.0f});
    float4 e0 = c.e0, e1 = c.e1, e2 = c.e2, e3 = c.e3;
    float4 cam = c.pos;
    if (U.slice_mode == 0u || U.slice_mode == 2u) {
        F3 n = normalized3(ld);  // past/future_light_ray_direction re-normalize (minkowski.rs:564-575)
        float4 base = U.slice_mode == 0u ? neg4(e0) : e0;
        *d = add4(add4(add4(base, mul4(e1, n.x)), mul4(e2, n.y)), mul4(e3, n.z));
        *o = U.slice_mode == 0u ? cam : sub4(cam, mul4(e0, U.frontier_view_offset));
    } else {
        *d = add4(add4(mul4(e1, ld.x), mul4(e2, ld.y)), mul4(e3, ld.z));
        *o = U.slice_mode == 3u ? add4(cam, mul4(e0, U.prophecy_delta)) : cam;
    }
    *sx_out = sx;
    *sy_out = sy;
}

// The star term of a pixel, brute force over every star as star_light does (star.rs:240-286).
// The pixel's footprint quantities of star_light (star.rs:240-253): the ray's spatial direction n,
// the footprint spread (RayFootprint::camera_pixel, star.rs:139-146) and the cone sign.
__device__ __forceinline__ void star_ray(const SrGpuUniforms& U, const Cam& cam, float4 d, float sx, float sy, float4* n,
                                         float* spread, float* cone) {
    float h = (float)U.size[1];
    float pitch = 2.0f * U.half_wh[1] / h;
    float inv_len = 1.0f / sqrtf(sx * sx + sy * sy + 1.0f);
    *spread = pitch * inv_len * sqrtf(inv_len);
    *cone = U.slice_mode == 0u ? -1.0f : (U.slice_mode == 2u ? 1.0f : 0.0f);
    *n = sub4(d, mul4(cam.e0, *cone));
}

static __device__ __noinline__ F3 stars_brute(const srk::SceneDev& s, const SrGpuUniforms& U, const Cam& cam, float4 o, float4 d,
                                       float sx, float sy, float lambda_max, const srk::BBConst& bbc) {
    float4 n;
    float spread, cone;
    star_ray(U, cam, d, sx, sy, &n, &spread, &cone);
    float4 e0 = cam.e0;
    BB bb{bbc.r5, bbc.g5, bbc.b5, bbc.wr, bbc.wg, bbc.wb};
    const float4* segs = s.stars + s.num_stars;
    F3 total{0.0f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < s.num_stars; ++i) {
        float4 hd = ld4(s.stars + i);
        float4 cd, cu;
        if (!cone_event(segs, __float_as_uint(hd.z), __float_as_uint(hd.w), o, e0, cone, &cd, &cu)) continue;
        F3 c;
        if (star_term(cd, cu, e0, cone, n, spread, lambda_max, hd.x, hd.y, bb, &c)) total = add(total, c);
    }
    return total;
}

}  // namespace srd
