// Device-side per-ray semantics of SpecRel's render path, shared by every render kernel.
//
// Each function evaluates in the operation order of the reference CPU renderer (the build uses
// --fmad=false and IEEE division / square root), so that with equal inputs the hit, lambda and
// tau are bit-identical to the reference and colours differ only through the last bits of the
// transcendentals (sinf, cosf, expf, atan2f, acosf):
//   intersect / slab test / safe_inv     mesh4d.rs:114-146, 175-211; bvh4d.rs:430-441
//   hit interpolation                    mesh4d.rs:382-425 over GpuAttr rows (gpu.rs:79-92)
//   shading, textures, lighting, sky     renderer.rs:414-1100
//   stars                                star.rs:162-286
// 4-vectors are float4 with .x = t, .y = x, .z = y, .w = z (the GPU layout of gpu.rs:37-40).
#pragma once
#include <cstdint>

#include "../../../include/specrel.h"

namespace srd {

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float a, float b, float c) { return F3{a, b, c}; }
__device__ __forceinline__ F3 add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 mul(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 mulv(F3 a, F3 b) { return F3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(F3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ F3 normalized3(F3 a) {
    float l = len3(a);
    if (l > 1e-12f) return mul(a, 1.0f / l);
    return F3{0.0f, 0.0f, 0.0f};
}

__device__ __forceinline__ float4 v4(float t, float x, float y, float z) { return make_float4(t, x, y, z); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
__device__ __forceinline__ float4 mul4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 neg4(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
__device__ __forceinline__ F3 spatial(float4 a) { return F3{a.y, a.z, a.w}; }
// Minkowski product <a, b> = -a.t b.t + a.x b.x + a.y b.y + a.z b.z (minkowski.rs:182-184).
__device__ __forceinline__ float mdot(float4 a, float4 b) { return -a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// Dual pairing alpha(v) (minkowski.rs:198-200).
__device__ __forceinline__ float edot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// Rust f32::rem_euclid (fmodf is exact).
__device__ __forceinline__ float rem_e(float x, float m) {
    float r = fmodf(x, m);
    return r < 0.0f ? r + fabsf(m) : r;
}
__device__ __forceinline__ float clampf_(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// rest_frame_cos (minkowski.rs:364-380).
__device__ __forceinline__ float rest_frame_cos(float4 v, float4 n, float4 u) {
    float4 vp = add4(v, mul4(u, mdot(v, u)));
    float l2 = mdot(vp, vp);
    if (l2 > 1e-12f) return clampf_(mdot(vp, n) / sqrtf(l2), -1.0f, 1.0f);
    return 0.0f;
}

// safe_inv_dir (bvh4d.rs:430-441).
__device__ __forceinline__ float safe_inv(float v) {
    if (fabsf(v) > 1e-12f) return 1.0f / v;
    return v >= 0.0f ? 1e12f : -1e12f;
}

// Aabb4D::intersect_ray (mesh4d.rs:114-146). Returns the entry parameter or -1 on a miss
// (t_min > 0 always, so a hit's entry is positive).
__device__ __forceinline__ float slab_enter(float4 bmin, float4 bmax, float4 o, float4 inv, float t_min, float t_max) {
    float t0 = (bmin.x - o.x) * inv.x, t1 = (bmax.x - o.x) * inv.x;
    float x0 = (bmin.y - o.y) * inv.y, x1 = (bmax.y - o.y) * inv.y;
    float y0 = (bmin.z - o.z) * inv.z, y1 = (bmax.z - o.z) * inv.z;
    float z0 = (bmin.w - o.w) * inv.w, z1 = (bmax.w - o.w) * inv.w;
    float en = fmaxf(fmaxf(fmaxf(fmaxf(t_min, fminf(t0, t1)), fminf(x0, x1)), fminf(y0, y1)), fminf(z0, z1));
    float ex = fminf(fminf(fminf(fminf(t_max, fmaxf(t0, t1)), fmaxf(x0, x1)), fmaxf(y0, y1)), fmaxf(z0, z1));
    return ex >= en ? en : -1.0f;
}

struct GeomHit {
    float lambda;
    float u, v, w;  // barycentrics (w0 = 1 - u - v - w)
};

// SimplexGeom4D::intersect_fast (mesh4d.rs:175-211) on the 80-byte hot record at `g`.
__device__ __forceinline__ bool intersect_geom(const float4* g, float4 o, float4 d, float t_min, float t_max, GeomHit* h) {
    float4 n = ld4(g + 1);
    float denom = edot(n, d);
    if (fabsf(denom) < 1e-9f) return false;
    float4 v0 = ld4(g + 0);
    float lambda = edot(n, sub4(v0, o)) / denom;
    if (lambda <= t_min || lambda >= t_max) return false;
    float4 ev = add4(o, mul4(d, lambda));
    float4 q = sub4(ev, v0);
    const float eps = -1e-5f;
    float u = edot(ld4(g + 2), q);
    if (u < eps || u > 1.0f - eps) return false;
    float v = edot(ld4(g + 3), q);
    if (v < eps || u + v > 1.0f - eps) return false;
    float w = edot(ld4(g + 4), q);
    if (w < eps || u + v + w > 1.0f - eps) return false;
    h->lambda = lambda;
    h->u = u;
    h->v = v;
    h->w = w;
    return true;
}

// Interpolated hit (HitRecord4D, mesh4d.rs:277-308, 382-425).
struct Hit {
    float lambda;
    float4 event;
    float b0, b1, b2, b3;  // tet barycentrics (w0, u, v, w)
    F3 tri_bary;
    float uv_u, uv_v;
    float tau;
    float grad_u, grad_v;
    float uvs_u, uvs_v;
    float4 normal, four_vel;
    float decided_at;
    uint32_t material;
};

__device__ __forceinline__ float bdot(float4 row, const Hit& h) {
    return row.x * h.b0 + row.y * h.b1 + row.z * h.b2 + row.w * h.b3;
}

// Simplex4D::interpolate_hit over the transposed cold record (12 rows of float4).
__device__ __forceinline__ void interpolate(const float4* a, float4 o, float4 d, const GeomHit& gh, Hit* h) {
    h->lambda = gh.lambda;
    h->event = add4(o, mul4(d, gh.lambda));
    h->b1 = gh.u;
    h->b2 = gh.v;
    h->b3 = gh.w;
    h->b0 = 1.0f - gh.u - gh.v - gh.w;
    h->uv_u = bdot(ld4(a + 0), *h);
    h->uv_v = bdot(ld4(a + 1), *h);
    h->tri_bary = F3{bdot(ld4(a + 2), *h), bdot(ld4(a + 3), *h), bdot(ld4(a + 4), *h)};
    h->tau = bdot(ld4(a + 5), *h);
    h->grad_u = bdot(ld4(a + 6), *h);
    h->grad_v = bdot(ld4(a + 7), *h);
    h->normal = ld4(a + 8);
    h->four_vel = ld4(a + 9);
    float4 misc = ld4(a + 10);
    h->uvs_u = misc.x;
    h->uvs_v = misc.y;
    h->material = __float_as_uint(misc.z);
    h->decided_at = bdot(ld4(a + 11), *h);
}

// ---------------------------------------------------------------------------------------------
// Shading (renderer.rs). `U` is the per-frame uniform block, `M` the material rows.
// ---------------------------------------------------------------------------------------------
struct Mat {
    F3 base, checker;
    float emission, grid, wire, cavity;
    uint32_t pattern;
};
__device__ __forceinline__ Mat load_mat(const float4* mats, uint32_t id) {
    float4 b = ld4(mats + 3 * id), c = ld4(mats + 3 * id + 1), p = ld4(mats + 3 * id + 2);
    Mat m;
    m.base = F3{b.x, b.y, b.z};
    m.emission = b.w;
    m.checker = F3{c.x, c.y, c.z};
    m.grid = c.w;
    m.wire = p.x;
    m.pattern = __float_as_uint(p.y);
    m.cavity = p.z;
    return m;
}

constexpr float PI_F = 3.14159265358979323846f;
constexpr float TAU_F = 6.28318530717958647692f;
constexpr float FRAC_1_PI_F = 0.318309886183790671537767526745028724f;

__device__ __forceinline__ F3 hsv_to_rgb(float h_deg, float s, float v) {  // renderer.rs:1081-1100
    float c = v * s;
    float h = rem_e(h_deg / 60.0f, 6.0f);
    float x = c * (1.0f - fabsf(rem_e(h, 2.0f) - 1.0f));
    float m = v - c;
    F3 r;
    if (h < 1.0f) r = F3{c, x, 0.0f};
    else if (h < 2.0f) r = F3{x, c, 0.0f};
    else if (h < 3.0f) r = F3{0.0f, c, x};
    else if (h < 4.0f) r = F3{0.0f, x, c};
    else if (h < 5.0f) r = F3{x, 0.0f, c};
    else r = F3{c, 0.0f, x};
    return F3{r.x + m, r.y + m, r.z + m};
}

__device__ __forceinline__ F3 shade_sky_gradient(float4 d) {  // renderer.rs:1056-1062
    F3 s = normalized3(spatial(d));
    float hz = clampf_(s.y * 0.5f + 0.5f, 0.0f, 1.0f);
    return add(mul(F3{0.12f, 0.16f, 0.25f}, 1.0f - hz), mul(F3{0.04f, 0.06f, 0.13f}, hz));
}
static __device__ __noinline__ F3 shade_sky(float4 d) {  // renderer.rs:1064-1079
    F3 s = normalized3(spatial(d));
    F3 sky = shade_sky_gradient(d);
    float theta = acosf(clampf_(s.y, -1.0f, 1.0f));
    float phi = atan2f(s.z, s.x);
    float gu = rem_e(phi / PI_F * 12.0f, 1.0f);
    float gv = rem_e(theta / PI_F * 6.0f, 1.0f);
    if (gu < 0.025f || gv < 0.025f) sky = add(sky, F3{0.06f, 0.09f, 0.14f});
    return sky;
}
__device__ __forceinline__ F3 apply_fog(F3 c, float4 d, float lambda) {  // renderer.rs:691-695
    float fog = expf(-0.008f * lambda);
    return add(mul(c, fog), mul(shade_sky_gradient(d), 1.0f - fog));
}

__device__ __forceinline__ bool point_on_hand(float dx, float dy, float ang, float len, float hw, float back) {
    float hx = sinf(ang), hy = cosf(ang);  // renderer.rs:930-943
    float along = dx * hx + dy * hy;
    float perp = fabsf(dx * hy - dy * hx);
    return along >= -back && along <= len && perp <= hw;
}

// sample_digital_tau (renderer.rs:946-981); glyph rows live after the LUT in `tables`.
static __device__ __noinline__ bool sample_digital_tau(float u, float v, float tau, const uint32_t* tables) {
    float rel_u = (u - 0.28f) / (0.72f - 0.28f);
    float rel_v = (0.18f - v) / (0.18f - 0.06f);
    float fc = floorf(rel_u * 35.0f), fr = floorf(rel_v * 7.0f);
    unsigned long long col = (fc > 0.0f) ? (unsigned long long)fc : 0ull;  // `as usize`
    unsigned long long row = (fr > 0.0f) ? (unsigned long long)fr : 0ull;
    if (col >= 35ull || row >= 7ull) return false;
    uint32_t ci = (uint32_t)col / 6u, cc = (uint32_t)col % 6u;
    if (ci >= 6u || cc >= 5u) return false;
    int t10 = (int)roundf(tau * 10.0f);  // saturating conversion, round half away from zero
    uint32_t at = t10 < 0 ? (uint32_t)(-(long long)t10) : (uint32_t)t10;
    uint32_t g;
    switch (ci) {
        case 0: g = t10 < 0 ? 11u : 10u; break;  // '-' : '+'
        case 1: g = (at / 100u) % 10u; break;
        case 2: g = (at / 10u) % 10u; break;
        case 3: g = 12u; break;                  // '.'
        case 4: g = at % 10u; break;
        default: g = 13u;                        // 'S'
    }
    return ((__ldg(tables + SR_GAMMA_LUT_SIZE + g * 7u + (uint32_t)row) >> (4u - cc)) & 1u) != 0u;
}

// The out-of-line helpers below take scalars by value: a struct passed by reference to a call
// would have to be stored to per-thread local memory first.
static __device__ __noinline__ F3 corner_mini_clock(float mdx, float mdy, float mr, float tau, F3 base) {
    if (mr > 0.080f) return mul(base, 1.15f);  // renderer.rs:880-927
    float ang = rem_e(atan2f(mdx, mdy), TAU_F);
    float fast = rem_e((tau / 1.0f) * TAU_F, TAU_F);
    float main = rem_e((tau / 10.0f) * TAU_F, TAU_F);
    F3 col{0.04f, 0.06f, 0.10f};
    if (ang <= fast && mr < 0.066f) col = add(col, mul(base, 0.25f));
    if (mr >= 0.062f && mr <= 0.078f) {
        float sector = ang / (TAU_F / 10.0f);
        float dist = fabsf(sector - roundf(sector));
        int tick = ((int)roundf(sector)) % 10;
        bool card = tick == 0 || tick == 5;
        float hw = card ? 0.13f : 0.07f;
        if (dist < hw) return tick == 0 ? F3{1.0f, 0.88f, 0.15f} : F3{0.80f, 0.85f, 0.92f};
    }
    if (point_on_hand(mdx, mdy, fast, 0.068f, 0.0065f, 0.008f)) return F3{0.25f, 0.98f, 1.0f};
    if (point_on_hand(mdx, mdy, main, 0.052f, 0.0085f, 0.008f)) return F3{1.0f, 0.95f, 0.30f};
    if (mr < 0.012f) return F3{1.0f, 1.0f, 1.0f};
    return col;
}

static __device__ __noinline__ F3 clock_face(float uv_u, float uv_v, float tau, float grad_u, float grad_v, float uvs_u,
                                             float uvs_v, float m_grid, F3 base, F3 checker, const uint32_t* tables) {
    float grid = fmaxf(m_grid, 1e-4f);  // renderer.rs:737-874
    float inv_grid = 1.0f / grid;
    float u = rem_e(uv_u * grid, 1.0f);
    float v = rem_e(uv_v * grid, 1.0f);
    // clock_tile_central_proper_time (renderer.rs:704-715)
    float ig2 = 1.0f / fmaxf(grid, 1e-4f);
    float central = tau - (((u - 0.5f) * ig2) * grad_u + ((v - 0.5f) * ig2) * grad_v);
    const float CX[4] = {0.135f, 0.865f, 0.135f, 0.865f}, CY[4] = {0.865f, 0.865f, 0.135f, 0.135f};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float mdx = u - CX[i], mdy = v - CY[i];
        float mr = sqrtf(mdx * mdx + mdy * mdy);
        if (mr <= 0.095f) {
            float osc = central + ((CX[i] - 0.5f) * inv_grid) * grad_u + ((CY[i] - 0.5f) * inv_grid) * grad_v;
            float px = (mdx * inv_grid) * uvs_u, py = (mdy * inv_grid) * uvs_v;
            float mrp = sqrtf(px * px + py * py);
            return corner_mini_clock(mdx, mdy, mr, osc - mrp, base);
        }
    }
    if (v >= 0.035f && v <= 0.205f && u >= 0.25f && u <= 0.75f) {
        if (!(v >= 0.050f && v <= 0.190f) || !(u >= 0.265f && u <= 0.735f)) return mul(base, 0.9f);
        if (v >= 0.06f && v <= 0.18f && u >= 0.28f && u <= 0.72f && sample_digital_tau(u, v, central, tables))
            return F3{1.0f, 0.96f, 0.30f};
        return F3{0.03f, 0.04f, 0.07f};
    }
    float dx = u - 0.50f, dy = v - 0.57f;
    float r = sqrtf(dx * dx + dy * dy);
    if (r > 0.330f) {
        int gu = (int)floorf(u * 4.0f), gv = (int)floorf(v * 4.0f);
        int s = (int)((unsigned)gu + (unsigned)gv);
        return ((s % 2 + 2) % 2) == 0 ? mul(base, 0.78f) : mul(checker, 0.78f);
    }
    if (r > 0.292f) return mul(base, 1.15f);
    float dxp = (dx * inv_grid) * uvs_u, dyp = (dy * inv_grid) * uvs_v;
    float rp = sqrtf(dxp * dxp + dyp * dyp);
    float dial = central - rp;
    float ang = rem_e(atan2f(dx, dy), TAU_F);
    float main = rem_e((dial / 10.0f) * TAU_F, TAU_F);
    F3 dc{0.04f, 0.06f, 0.10f};
    if (ang <= main && r < 0.236f) dc = add(dc, mul(base, 0.22f));
    if (r >= 0.220f && r <= 0.286f) {
        float sector = ang / (TAU_F / 10.0f);
        float dist = fabsf(sector - roundf(sector));
        int tick = ((int)roundf(sector)) % 10;
        bool card = tick == 0 || tick == 5;
        float hw = card ? 0.105f : 0.055f;
        float inner = card ? 0.218f : 0.242f;
        if (dist < hw && r >= inner) {
            if (tick == 0) return F3{1.0f, 0.88f, 0.15f};
            if (card) return F3{1.0f, 1.0f, 1.0f};
            return F3{0.75f, 0.80f, 0.88f};
        }
    }
    float fast = rem_e((dial / 1.0f) * TAU_F, TAU_F);
    if (point_on_hand(dx, dy, fast, 0.254f, 0.012f, 0.025f)) return F3{0.25f, 0.98f, 1.0f};
    if (point_on_hand(dx, dy, main, 0.228f, 0.022f, 0.025f)) return F3{1.0f, 0.95f, 0.30f};
    if (point_on_hand(dx, dy, main, 0.236f, 0.030f, 0.025f)) return F3{0.02f, 0.02f, 0.04f};
    float slow = rem_e((dial / 100.0f) * TAU_F, TAU_F);
    if (point_on_hand(dx, dy, slow, 0.162f, 0.026f, 0.025f)) return F3{1.0f, 0.35f, 0.25f};
    if (r < 0.034f) return F3{1.0f, 1.0f, 1.0f};
    return dc;
}

static __device__ __noinline__ F3 light_clock(float uv_u, float uv_v, float tau, float m_grid, float m_cavity, F3 base) {
    float u = rem_e(uv_u * m_grid, 1.0f);  // renderer.rs:988-1052
    float v = rem_e(uv_v * m_grid, 1.0f);
    if (!(u >= 0.12f && u <= 0.88f)) return mul(base, 0.65f);
    if ((v >= 0.04f && v <= 0.10f) || (v >= 0.90f && v <= 0.96f)) return F3{0.75f, 0.90f, 0.98f};
    if (!(v >= 0.10f && v <= 0.90f)) return F3{0.08f, 0.12f, 0.16f};
    float period = fmaxf(2.0f * m_cavity, 1e-4f);
    float cycle = rem_e(tau / period, 1.0f);
    float bounce = cycle < 0.5f ? cycle * 2.0f : (1.0f - cycle) * 2.0f;
    float pv = 0.10f + 0.80f * bounce;
    float dv = fabsf(v - pv), du = fabsf(u - 0.5f);
    float dist = sqrtf(du * du * 0.7f + dv * dv);
    F3 col{0.05f, 0.09f, 0.13f};
    float ruler = rem_e((v - 0.10f) / 0.80f * 8.0f, 1.0f);
    if ((u < 0.22f || u > 0.78f) && ruler < 0.08f) col = add(col, F3{0.20f, 0.35f, 0.35f});
    if (du < 0.015f) col = add(col, F3{0.06f, 0.16f, 0.16f});
    if (dv < 0.032f) {
        float k = 1.0f - dv / 0.032f;
        col = add(col, mul(base, 0.9f * (k * k)));
    }
    if (dist < 0.11f) {
        float k = 1.0f - dist / 0.11f;
        col = add(col, mul(F3{1.0f, 1.0f, 0.85f}, 1.4f * (k * k)));
    }
    return col;
}

__device__ __forceinline__ F3 surface_albedo(const Hit& h, const Mat& m, const uint32_t* tables) {
    F3 a;  // renderer.rs:544-580
    if (m.pattern == 0u) {
        int gu = (int)floorf(h.uv_u * m.grid), gv = (int)floorf(h.uv_v * m.grid);
        int s = (int)((unsigned)gu + (unsigned)gv);
        F3 col = ((s % 2 + 2) % 2) == 0 ? m.base : m.checker;
        float mt = fminf(fminf(h.tri_bary.x, h.tri_bary.y), h.tri_bary.z);
        if (mt < m.wire) {
            float et = clampf_(mt / m.wire, 0.0f, 1.0f);
            col = add(mul(F3{0.07f, 0.07f, 0.07f}, 1.0f - et), mul(col, et));
        }
        a = col;
    } else if (m.pattern == 1u) {
        a = clock_face(h.uv_u, h.uv_v, h.tau, h.grad_u, h.grad_v, h.uvs_u, h.uvs_v, m.grid, m.base, m.checker, tables);
    } else {
        a = light_clock(h.uv_u, h.uv_v, h.tau, m.grid, m.cavity, m.base);
    }
    if (m.pattern != 0u) {
        float ut = rem_e(h.uv_u * m.grid, 1.0f), vt = rem_e(h.uv_v * m.grid, 1.0f);
        float border = fminf(fminf(ut, 1.0f - ut), fminf(vt, 1.0f - vt));
        if (border < 0.025f) a = mul(a, 0.35f);
    }
    return a;
}

__device__ __forceinline__ F3 decision_age_color(float age) {  // renderer.rs:494-507
    if (age < 0.0f) return F3{0.14f, 0.14f, 0.18f};
    F3 col = hsv_to_rgb(fminf(age * 4.0f, 240.0f), 0.82f, 0.88f);
    if (age < 0.45f) {
        float f = 1.0f - age / 0.45f;
        col = add(mul(col, 1.0f - f * 0.7f), mul(F3{1.0f, 0.96f, 0.65f}, f * 0.9f));
    }
    if (fabsf(rem_e(age * 0.5f, 1.0f) - 0.5f) > 0.465f) col = F3{0.95f, 0.98f, 1.0f};
    return col;
}

static __device__ __noinline__ F3 apply_haze(F3 base, float4 ev, const SrGpuUniforms& U) {  // renderer.rs:514-541
    const float SHELL = 0.18f;
    float inside = -INFINITY;
    for (uint32_t i = 0; i < U.num_haze; ++i) {
        float4 o = v4(U.haze_origin[i][0], U.haze_origin[i][1], U.haze_origin[i][2], U.haze_origin[i][3]);
        float4 d = sub4(ev, o);
        inside = fmaxf(inside, d.x - len3(spatial(d)));
    }
    if (inside <= -SHELL) return base;
    F3 col = base;
    if (fabsf(inside) < SHELL) {
        float k = 1.0f - fabsf(inside) / SHELL;
        col = add(col, mul(F3{0.45f, 0.92f, 1.0f}, 0.85f * k * k));
    }
    if (inside > 0.0f) {
        float ripple = 0.5f + 0.5f * sinf(ev.y * 3.5f + ev.w * 3.5f - ev.x * 4.0f) * cosf(inside * 5.0f);
        F3 haze = add(mul(F3{0.32f, 0.18f, 0.62f}, 1.0f - 0.35f * ripple), mul(F3{0.18f, 0.72f, 0.92f}, 0.35f * ripple));
        float alpha = 0.55f + 0.25f * fminf(inside * 0.5f, 1.0f);
        col = add(mul(col, 1.0f - alpha), mul(haze, alpha));
    }
    return col;
}

__device__ __forceinline__ float4 u_e(const SrGpuUniforms& U, int a) { return v4(U.e[a][0], U.e[a][1], U.e[a][2], U.e[a][3]); }

// The observer of a frame: from the uniform block, or (FP64 path) from the device buffer the
// camera kernel wrote (event rebased to the scene anchor, tetrad rounded from double).
struct Cam {
    float4 pos, e0, e1, e2, e3, frontier;
};
__device__ __forceinline__ Cam load_cam(const SrGpuUniforms& U, const float4* cam_dev) {
    Cam c;
    if (cam_dev) {
        c.pos = cam_dev[0];
        c.e0 = cam_dev[1];
        c.e1 = cam_dev[2];
        c.e2 = cam_dev[3];
        c.e3 = cam_dev[4];
        c.frontier = cam_dev[5];
    } else {
        c.pos = v4(U.cam_pos[0], U.cam_pos[1], U.cam_pos[2], U.cam_pos[3]);
        c.e0 = u_e(U, 0);
        c.e1 = u_e(U, 1);
        c.e2 = u_e(U, 2);
        c.e3 = u_e(U, 3);
        c.frontier = v4(U.frontier_origin[0], U.frontier_origin[1], U.frontier_origin[2], U.frontier_origin[3]);
    }
    return c;
}

// light_emission_event (renderer.rs:585-606): the direction to the light and the distance.
__device__ __forceinline__ void light_ray(const SrGpuUniforms& U, const Cam& cam, float4 ev, float4* to_light, float* dist) {
    F3 lp{U.light_pos[1], U.light_pos[2], U.light_pos[3]};
    F3 tl = sub(lp, spatial(ev));
    float dl = fmaxf(len3(tl), 1e-4f);
    float t_emit;
    if (U.shadow_mode == 2u) {
        // camera beta = e0.spatial / e0.t, divided as Vec3 / f32 does (minkowski.rs:274-280)
        float4 e0 = cam.e0;
        F3 beta = fabsf(e0.x) > 1e-12f ? mul(spatial(e0), 1.0f / e0.x) : F3{0.0f, 0.0f, 0.0f};
        t_emit = ev.x + dot3(beta, tl);
    } else {
        t_emit = ev.x - dl;
    }
    float4 emit = v4(t_emit, lp.x, lp.y, lp.z);
    *to_light = mul4(sub4(emit, ev), 1.0f / dl);
    *dist = dl;
}

// ---------------------------------------------------------------------------------------------
// Stars (star.rs).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float planck(float lam_pow5, float lam, float temp) {
    float x = fminf(14388.0f / (lam * fmaxf(temp, 1.0f)), 80.0f);
    return 1.0f / (lam_pow5 * (expf(x) - 1.0f));
}
// powi(5) of the three primaries and the white-point Planck values come from the host.
struct BB {
    float r5, g5, b5, wr, wg, wb;
};
__device__ __forceinline__ F3 blackbody_rgb(float temp, const BB& bb) {
    return F3{planck(bb.r5, 0.610f, temp) / bb.wr, planck(bb.g5, 0.550f, temp) / bb.wg, planck(bb.b5, 0.465f, temp) / bb.wb};
}

struct StarHeader {
    float temp, cn;
    uint32_t first, count;
};

__device__ __forceinline__ float past_the_cone(float4 ev, float4 o, float4 e0, float cone) {
    float4 d = sub4(ev, o);
    float tau = -mdot(d, e0);
    if (cone == 0.0f) return tau;
    float rho = sqrtf(fmaxf(mdot(d, d) + tau * tau, 0.0f));
    return tau - cone * rho;
}
__device__ __forceinline__ float segment_cone_crossing(float4 ev, float4 u, float4 o, float4 e0, float cone) {
    float4 d0 = sub4(ev, o);
    if (cone == 0.0f) {
        float tau0 = -mdot(d0, e0);
        float g = -mdot(u, e0);
        return -tau0 / g;
    }
    float a = mdot(d0, d0);
    float b = mdot(d0, u);
    float sq = sqrtf(fmaxf(b * b + a, 0.0f));
    if (cone < 0.0f) return b > 0.0f ? -a / (b + sq) : b - sq;
    return b < 0.0f ? -a / (b - sq) : b + sq;
}
// worldline_cone_event (star.rs:228-235): `segs` = the packed segments (3 float4 each).
__device__ __forceinline__ bool cone_event(const float4* segs, uint32_t first, uint32_t count, float4 o, float4 e0,
                                           float cone, float4* d_out, float4* u_out) {
    if (count == 0u) return false;
    uint32_t lo = 0, hi = count;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (past_the_cone(ld4(segs + 3u * (first + mid)), o, e0, cone) <= 0.0f) lo = mid + 1u;
        else hi = mid;
    }
    uint32_t k = first + (lo > 1u ? lo : 1u) - 1u;
    float4 ev = ld4(segs + 3u * k), u = ld4(segs + 3u * k + 1u), rg = ld4(segs + 3u * k + 2u);
    float s = segment_cone_crossing(ev, u, o, e0, cone);
    if (!(s >= rg.x && s <= rg.y)) return false;
    *d_out = add4(sub4(ev, o), mul4(u, s));
    *u_out = u;
    return true;
}

// The contribution of one star whose cone event is (d, u) to the ray `n` (star.rs:254-283).
__device__ __forceinline__ bool star_term(float4 d, float4 u, float4 e0, float cone, float4 n, float spread,
                                          float lambda_max, float temp, float cn, const BB& bb, F3* out) {
    float tau = -mdot(d, e0);
    float4 r = add4(d, mul4(e0, -tau));
    float along = mdot(r, n);
    if (along <= 0.0f || along >= lambda_max) return false;
    float4 perp = sub4(r, mul4(n, along));
    float d2 = fmaxf(mdot(perp, perp), 0.0f);
    float sigma = 0.6f * (0.0f + spread * along);
    float cut = 4.0f * sigma;
    if (d2 >= cut * cut) return false;
    float inv = 1.0f / (2.0f * sigma * sigma);
    float kernel = expf(-d2 * inv) * inv * FRAC_1_PI_F;
    float dop = 1.0f;
    if (cone < 0.0f) {
        float lam = sqrtf(fmaxf(mdot(r, r), 0.0f));
        float du = mdot(d, u);
        if (du > 0.0f) dop = lam / du;
    }
    *out = mul(blackbody_rgb(temp * dop, bb), cn * kernel);
    return true;
}

}  // namespace srd
