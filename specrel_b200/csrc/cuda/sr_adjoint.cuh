// The gradient of an image loss with respect to the observer (no counterpart kernel in the
// reference; SpecRel renders forward only).
//
//   loss = sum over pixels and r, g, b of (P_L(HDR) - P_L(target))^2 on the linear pre-bloom HDR
//          image, P_L = L halvings by 2x2 box averages (L = 0: the image itself; coarse levels
//          widen the loss's basin for a coarse-to-fine descent)
//   theta = (rapidity x, y, z, event t, x, y, z) of Tetrad::rest().boost_local(rapidity)
//
// The forward frame is rendered first; its discrete outcomes are held fixed: which tetrahedron each
// ray hits, the shadow tests, the texture lookups (albedo), the sky's grid lines, which segment of a
// star's worldline crosses the cone and which stars pass the footprint cut. Everything smooth between
// theta and the HDR colour is differentiated in forward mode (7 tangents, sr_dual.cuh): the FP64
// tetrad and its rapidity derivatives, the camera ray, the hit parameter on the tetrahedron's
// hyperplane and the hit event, the light direction and distance of the null (or camera-slice)
// emission event, the rest-frame Lambert and view cosines, the attenuation, the distance fog, the
// sky gradient, and for every star its cone crossing, footprint kernel, Doppler factor and
// blackbody colour. Traversal is not stored: the hit slots of the forward frame identify the
// tetrahedra. Per-pixel sums are accumulated in double per block and reduced in a fixed order.
// Included by sr_fast.cu after sr_stars.cuh.
#pragma once
#include "sr_dual.cuh"

namespace srg {

// boost_local at zero rapidity: the value stays the rest tetrad; the derivative is the boost
// generator, d e0 / d phi_j = e_j and d e_j / d phi_j = e0 (a boost mixes e0 and e_j).
__device__ __forceinline__ void zero_boost_tangent(srk::D4T<DD3>* e, const DD3& rx, const DD3& ry, const DD3& rz) {
    const DD3 r[3] = {rx, ry, rz};
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
            const double g = r[j].d[k];  // d phi_j / d phi_k
            if (g == 0.0) continue;
            srk::D4T<DD3>& e0 = e[0];
            srk::D4T<DD3>& ej = e[1 + j];
            const double e0c[4] = {e0.t.v, e0.x.v, e0.y.v, e0.z.v}, ejc[4] = {ej.t.v, ej.x.v, ej.y.v, ej.z.v};
            e0.t.d[k] += g * ejc[0];
            e0.x.d[k] += g * ejc[1];
            e0.y.d[k] += g * ejc[2];
            e0.z.d[k] += g * ejc[3];
            ej.t.d[k] += g * e0c[0];
            ej.x.d[k] += g * e0c[1];
            ej.y.d[k] += g * e0c[2];
            ej.z.d[k] += g * e0c[3];
        }
}

// The camera as duals: event (anchor-relative) and e0..e3.
struct DCam {
    DF4 pos, e[4];
};

// rest_frame_cos (minkowski.rs:364-380) of a varying vector against a fixed normal and velocity.
__device__ __forceinline__ DF rest_frame_cos(const DF4& v, float4 n, float4 u) {
    DF4 vp = add4(v, mul4(u, mdot(v, u)));
    DF l2 = mdot(vp, vp);
    if (l2.v > 1e-12f) return dclamp(mdot(vp, n) / dsqrt(l2), -1.0f, 1.0f);
    return dconst(0.0f);
}

__device__ __forceinline__ DF3 sky_gradient(const DF4& d) {  // renderer.rs:1056-1062
    DF3 s = normalized3(spatial(d));
    DF hz = dclamp(s.y * 0.5f + 0.5f, 0.0f, 1.0f);
    return add(mul(F3{0.12f, 0.16f, 0.25f}, 1.0f - hz), mul(F3{0.04f, 0.06f, 0.13f}, hz));
}

__device__ __forceinline__ DF planck(float lam_pow5, float lam, const DF& temp) {
    DF x = dminc(14388.0f / (lam * dmaxc(temp, 1.0f)), 80.0f);
    return 1.0f / (lam_pow5 * (dexp(x) - 1.0f));
}

}  // namespace srg

namespace srk {

using namespace srg;

struct AdjointArgs {
    SceneDev s;
    const SrGpuUniforms* U;   // the observer's uniform block (device)
    const ObsDev* obs;
    const uint32_t* star_pre;
    const DCam* dcam;
    const float4* hits;
    const uint32_t* slots;
    const uint8_t* shadow;
    const DF4* star_dcd;      // per star: the cone event offset as duals
    const float4* star_cu;    // per star: the crossing segment's 4-velocity (forward pass)
    const uint32_t* count;
    const uint32_t* offset;
    const uint32_t* list;
    uint32_t list_cap;
    uint32_t stars_on;
    const float4* hdr_fwd;    // the forward frame's HDR (level 0)
    const double* weight;     // W*H*3: d loss / d HDR (r, g, b)
    double* partials;         // per block: -, grad[7], primal mismatches, star terms
    BBConst bb;
    // The discrete outcomes besides the hits: sky grid line per pixel, and per (sorted star-list
    // entry, pixel of its tile) whether the star's term passed the footprint cut.
    uint8_t* grid;
    uint32_t* pass;           // 8 words (256 bits) per list entry
    uint32_t frozen;          // 0: gradient, recording the outcomes; 1: values under the recorded outcomes
    float4* hdr_out;          // frozen: the HDR values (W*H)
    uint32_t y0, y1;          // the pixel rows of this call (a band of the frame, or all of it)
    uint32_t tile0;           // the first 16x16 tile of the launch (blocks take tile0, tile0 + 1, ...)
};
constexpr int ADJ_SLOTS = 10;

// The camera's duals from the FP64 observer: TetradT<DD3> carries the rapidity derivatives; the
// event's derivative is the identity.
__global__ void k_adjoint_camera(SrCameraF64 c, double a0, double a1, double a2, double a3, DCam* out) {
    DD3 r[3] = {DD3(c.rapidity[0]), DD3(c.rapidity[1]), DD3(c.rapidity[2])};
    for (int k = 0; k < 3; ++k) r[k].d[k] = 1.0;
    TetradT<DD3> t;
    t.observer(r[0], r[1], r[2], c.yaw, c.pitch, c.roll);
    DCam dc;
    const double anchor[4] = {a0, a1, a2, a3};
    DF* pos[4] = {&dc.pos.x, &dc.pos.y, &dc.pos.z, &dc.pos.w};
    for (int k = 0; k < 4; ++k) {
        *pos[k] = dconst((float)(c.event[k] - anchor[k]));
        pos[k]->d[3 + k] = 1.0f;
    }
    for (int a = 0; a < 4; ++a) {
        const DD3* comp[4] = {&t.e[a].t, &t.e[a].x, &t.e[a].y, &t.e[a].z};
        DF* dst[4] = {&dc.e[a].x, &dc.e[a].y, &dc.e[a].z, &dc.e[a].w};
        for (int k = 0; k < 4; ++k) {
            *dst[k] = dconst((float)comp[k]->v);
            for (int j = 0; j < 3; ++j) dst[k]->d[j] = (float)comp[k]->d[j];
        }
    }
    *out = dc;
}

// Each star's cone event as duals (past light cone, observer 0): the crossing segment found by the
// forward pass's binary search, the crossing parameter and the event offset differentiated.
__global__ void __launch_bounds__(128) k_adjoint_stars(const float4* stars, uint32_t num_stars, const DCam* dcam,
                                                       DF4* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num_stars) return;
    const DCam& c = *dcam;
    const float4 o = val4(c.pos), e0 = val4(c.e[0]);
    const float4* segs = stars + num_stars;
    const float4 hd = __ldg(stars + i);
    const uint32_t first = __float_as_uint(hd.z), count = __float_as_uint(hd.w);
    if (count == 0u) return;
    uint32_t lo = 0, hi = count;
    while (lo < hi) {  // cone_event's search (star.rs:228-235)
        uint32_t mid = (lo + hi) / 2u;
        if (past_the_cone(__ldg(segs + 3u * (first + mid)), o, e0, -1.0f) <= 0.0f) lo = mid + 1u;
        else hi = mid;
    }
    const uint32_t k = first + (lo > 1u ? lo : 1u) - 1u;
    const float4 ev = __ldg(segs + 3u * k), u = __ldg(segs + 3u * k + 1u);
    // segment_cone_crossing, past cone.
    const DF4 d0 = sub4(ev, c.pos);
    const DF a = mdot(d0, d0), b = mdot(d0, u);
    const DF sq = dsqrt(dmaxc(b * b + a, 0.0f));
    const DF s = b.v > 0.0f ? -a / (b + sq) : b - sq;
    out[i] = add4(sub4(ev, c.pos), mul4(u, s));
}

// One 16x16 tile per block, as k_star_tiles: the tile's star list sorted by index, then per pixel
// the dual HDR colour, its residual against the target and the partial sums.
__global__ void __launch_bounds__(256) k_adjoint_pixels(AdjointArgs a) {
    extern __shared__ uint32_t keys[];
    __shared__ double red[ADJ_SLOTS][8];
    __shared__ int bad;
    const uint32_t tile = a.tile0 + blockIdx.x;
    const ObsDev& od = a.obs[0];
    const SrGpuUniforms& U = a.U[0];
    const uint32_t tx16 = (od.width + STAR_TILE - 1) / STAR_TILE;
    const uint32_t px = (tile % tx16) * STAR_TILE + threadIdx.x % STAR_TILE;
    const uint32_t py = (tile / tx16) * STAR_TILE + threadIdx.x / STAR_TILE;
    const bool inside = px < od.width && py < od.height && py >= a.y0 && py < a.y1;
    uint32_t cnt = 0;
    bool brute = false;
    if (a.stars_on) {
        cnt = a.count[tile];
        const uint32_t off = a.offset[tile];
        brute = cnt > STAR_SORT_CAP || (uint64_t)off + cnt > a.list_cap;
        if (!brute) {
            uint32_t p2 = 1;
            while (p2 < cnt) p2 <<= 1;
            if (threadIdx.x == 0) bad = 0;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) {
                const uint32_t v = k < cnt ? a.list[off + k] : 0xFFFFFFFFu;
                if (k < cnt && v >= a.s.num_stars) bad = 1;
                keys[k] = v;
            }
            __syncthreads();
            brute = bad != 0;
            if (!brute)
                for (uint32_t size = 2; size <= p2; size <<= 1)
                    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                        for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) {
                            const uint32_t j = k ^ stride;
                            if (j > k) {
                                const bool up = (k & size) == 0;
                                const uint32_t x = keys[k], y = keys[j];
                                if ((x > y) == up) {
                                    keys[k] = y;
                                    keys[j] = x;
                                }
                            }
                        }
                        __syncthreads();
                    }
        }
    }
    double acc[ADJ_SLOTS];
    for (int k = 0; k < ADJ_SLOTS; ++k) acc[k] = 0.0;
    if (inside) {
        const DCam& dc = *a.dcam;
        // The camera ray of the past light cone (camera_ray): d = -e0 + n.x e1 + n.y e2 + n.z e3.
        const float w = (float)U.size[0], h = (float)U.size[1];
        const float ndc_y = 1.0f - 2.0f * (((float)py + 0.5f) / h);
        const float ndc_x = 2.0f * (((float)px + 0.5f) / w) - 1.0f;
        const float sx = ndc_x * U.half_wh[0], sy = ndc_y * U.half_wh[1];
        const F3 n3 = srd::normalized3(srd::normalized3(F3{sx, sy, 1.0f}));
        const DF4 d = add4(add4(add4(neg4(dc.e[0]), mul4(dc.e[1], n3.x)), mul4(dc.e[2], n3.y)), mul4(dc.e[3], n3.z));
        const DF4& o = dc.pos;
        const uint32_t l = py * od.width + px, p = od.pix_base + l;
        const uint32_t slot = a.slots[p];
        DF3 color;
        float lambda_max = INFINITY;
        bool primal_ok = true;
        if (slot != 0xFFFFFFFFu) {
            const float4* g = a.s.geoms + 5u * slot;
            const float4 nrm = __ldg(g + 1), v0 = __ldg(g);
            const DF lam = edot(nrm, sub4(v0, o)) / edot(nrm, d);
            const float4 hr = a.hits[p];
            primal_ok = a.frozen || lam.v == hr.x;
            lambda_max = hr.x;
            const DF4 ev = add4(o, mul4(d, lam));
            // The forward hit record (fixed barycentrics) gives the albedo, normal, velocity, material.
            Hit hit;
            srd::interpolate(a.s.attrs + 12u * slot, val4(o), val4(d), GeomHit{hr.x, hr.y, hr.z, hr.w}, &hit);
            const Mat m = load_mat(a.s.mats, hit.material);
            const F3 albedo = surface_albedo(hit, m, a.s.tables);
            // light_emission_event (renderer.rs:585-606).
            const DF3 tl{U.light_pos[1] - ev.y, U.light_pos[2] - ev.z, U.light_pos[3] - ev.w};
            const DF dl = dmaxc(len3(tl), 1e-4f);
            DF t_emit;
            if (U.shadow_mode == 2u) {
                const DF4& e0 = dc.e[0];
                const DF3 beta = fabsf(e0.x.v) > 1e-12f ? mul(spatial(e0), 1.0f / e0.x) : DF3{dconst(0.0f), dconst(0.0f), dconst(0.0f)};
                t_emit = ev.x + dot3(beta, tl);
            } else {
                t_emit = ev.x - dl;
            }
            const DF4 emit{t_emit, dconst(U.light_pos[1]), dconst(U.light_pos[2]), dconst(U.light_pos[3])};
            const DF4 to_light = mul4(sub4(emit, ev), 1.0f / dl);
            // compute_illumination (renderer.rs:609-653) with the forward shadow result.
            const DF cl = dmaxc(rest_frame_cos(to_light, hit.normal, hit.four_vel), 0.0f);
            const DF cv = dmaxc(-rest_frame_cos(d, hit.normal, hit.four_vel), 0.0f);
            DF lighting;
            if (m.pattern == 0u) {
                const bool in_shadow = cl.v > 0.0f && U.shadow_mode != 0u && a.shadow[p] == 2;
                const float sf = in_shadow ? 0.32f : 1.0f;
                const DF atten = 1.0f / (1.0f + 0.006f * dl * dl);
                lighting = m.emission + 0.30f * cv + 0.80f * sf * cl * atten;
            } else {
                lighting = 0.72f + 0.38f * cv + 0.22f * cl;
            }
            const DF3 lit = mul(albedo, lighting);
            const DF fog = dexp(-0.008f * lam);
            color = add(mul(lit, fog), mul(sky_gradient(d), 1.0f - fog));
        } else {
            color = sky_gradient(d);
            bool grid;
            if (a.frozen) {
                grid = a.grid[l] != 0;
            } else {
                const F3 sv = shade_sky(val4(d)), gv = shade_sky_gradient(val4(d));
                grid = sv.x != gv.x || sv.y != gv.y || sv.z != gv.z;
                a.grid[l] = grid ? 1 : 0;
            }
            if (grid) {  // the grid lines: a constant
                color.x = color.x + 0.06f;
                color.y = color.y + 0.09f;
                color.z = color.z + 0.14f;
            }
        }
        if (a.stars_on && !brute) {
            const float inv_len = 1.0f / sqrtf(sx * sx + sy * sy + 1.0f);
            const float spread = (2.0f * U.half_wh[1] / h) * inv_len * sqrtf(inv_len);
            const DF4& e0 = dc.e[0];
            const DF4 n = sub4(d, mul4(e0, -1.0f));
            DF3 total = dconst3(F3{0.0f, 0.0f, 0.0f});
            const uint32_t off = a.offset[tile];
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t i = keys[k];
                const DF4 cd = a.star_dcd[i];
                uint32_t* word = a.pass + (size_t)(off + k) * 8u + (threadIdx.x >> 5);
                const uint32_t bit = 1u << (threadIdx.x & 31u);
                if (a.frozen && !(*word & bit)) continue;
                // star_term (star.rs:254-283).
                const DF tau = -mdot(cd, e0);
                const DF4 r = add4(cd, mul4(e0, -tau));
                const DF along = mdot(r, n);
                if (!a.frozen && (along.v <= 0.0f || along.v >= lambda_max)) continue;
                const DF4 perp = sub4(r, mul4(n, along));
                const DF d2 = dmaxc(mdot(perp, perp), 0.0f);
                const DF sigma = 0.6f * (0.0f + spread * along);
                const DF cut = 4.0f * sigma;
                if (!a.frozen) {
                    if (d2.v >= cut.v * cut.v) continue;
                    atomicOr(word, bit);
                }
                const DF inv = 1.0f / (2.0f * sigma * sigma);
                const DF kernel = dexp(-d2 * inv) * inv * FRAC_1_PI_F;
                DF dop = dconst(1.0f);
                const DF lamr = dsqrt(dmaxc(mdot(r, r), 0.0f));
                const DF du = mdot(cd, __ldg(a.star_cu + i));
                if (du.v > 0.0f) dop = lamr / du;
                const float4 hd = __ldg(a.s.stars + i);
                const DF temp = hd.x * dop;
                const DF sc = hd.y * kernel;
                const DF3 c{planck(a.bb.r5, 0.610f, temp) / a.bb.wr * sc, planck(a.bb.g5, 0.550f, temp) / a.bb.wg * sc,
                            planck(a.bb.b5, 0.465f, temp) / a.bb.wb * sc};
                total = add(total, c);
                acc[9] += 1.0;
            }
            color = add(color, total);
        }
        if (a.frozen) {
            a.hdr_out[l] = make_float4(color.x.v, color.y.v, color.z.v, 0.0f);
        } else {
            const float4 fw = a.hdr_fwd[(size_t)od.pyr_base + l];
            primal_ok = primal_ok && color.x.v == fw.x && color.y.v == fw.y && color.z.v == fw.z;
        }
        if (!primal_ok || (a.stars_on && brute)) acc[8] += 1.0;
        const DF* ch[3] = {&color.x, &color.y, &color.z};
        for (int c = 0; c < 3; ++c) {
            const double wc = a.weight[3ull * l + c];
            for (int k = 0; k < NT; ++k) acc[1 + k] += wc * (double)ch[c]->d[k];
        }
    }
    // Fixed-order block reduction: within each warp, then over the 8 warps.
    for (int k = 0; k < ADJ_SLOTS; ++k)
        for (int off = 16; off > 0; off >>= 1) acc[k] += __shfl_down_sync(0xFFFFFFFFu, acc[k], off);
    if ((threadIdx.x & 31u) == 0)
        for (int k = 0; k < ADJ_SLOTS; ++k) red[k][threadIdx.x >> 5] = acc[k];
    __syncthreads();
    if (threadIdx.x < ADJ_SLOTS) {
        double t = 0.0;
        for (int wi = 0; wi < 8; ++wi) t += red[threadIdx.x][wi];
        a.partials[(size_t)blockIdx.x * ADJ_SLOTS + threadIdx.x] = t;
    }
}

// One level of the loss's image pyramid: 2x2 box averages, taps clamped at odd edges.
__global__ void k_adj_down(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dw || y >= dh) return;
    const uint32_t x0 = 2u * x, x1 = min(2u * x + 1u, sw - 1u), y0 = 2u * y, y1 = min(2u * y + 1u, sh - 1u);
    const float4 a = src[(size_t)y0 * sw + x0], b = src[(size_t)y0 * sw + x1];
    const float4 c = src[(size_t)y1 * sw + x0], d = src[(size_t)y1 * sw + x1];
    dst[(size_t)y * dw + x] = make_float4(((a.x + b.x) + (c.x + d.x)) * 0.25f, ((a.y + b.y) + (c.y + d.y)) * 0.25f,
                                          ((a.z + b.z) + (c.z + d.z)) * 0.25f, 0.0f);
}

// The transpose of k_adj_down on the loss weights (3 doubles per pixel): source pixel (x', y')
// feeds only destination (x'/2, y'/2), twice along an axis whose last tap was clamped onto it.
__global__ void k_adj_up(const double* gd, uint32_t dw, uint32_t dh, double* gs, uint32_t sw, uint32_t sh) {
    const uint32_t xs = blockIdx.x * blockDim.x + threadIdx.x, ys = blockIdx.y * blockDim.y + threadIdx.y;
    if (xs >= sw || ys >= sh) return;
    const uint32_t x = xs / 2u, y = ys / 2u;
    const double wx = (xs == 2u * x && 2u * x + 1u >= sw) ? 2.0 : 1.0;
    const double wy = (ys == 2u * y && 2u * y + 1u >= sh) ? 2.0 : 1.0;
    const double k = 0.25 * wx * wy;
    for (int c = 0; c < 3; ++c) gs[((size_t)ys * sw + xs) * 3 + c] = k * gd[((size_t)y * dw + x) * 3 + c];
}

// Residual of the chosen level: the loss's per-block partial sums and its weights 2 (P - T).
// The residual of the loss level's pixels in rows [r0, r1) (width w): the loss terms and their
// weights; pixels outside the band weigh nothing.
__global__ void __launch_bounds__(256) k_adj_residual(const float4* p, const float4* t, uint32_t n, uint32_t w,
                                                      uint32_t r0, uint32_t r1, double* weight, double* partials) {
    __shared__ double red[8];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (i < n) {
        const uint32_t row = i / w;
        const bool in_band = row >= r0 && row < r1;
        const float4 a = p[i], b = t[i];
        const double r[3] = {(double)a.x - (double)b.x, (double)a.y - (double)b.y, (double)a.z - (double)b.z};
        for (int c = 0; c < 3; ++c) {
            if (in_band) acc += r[c] * r[c];
            weight[3ull * i + c] = in_band ? 2.0 * r[c] : 0.0;
        }
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, off);
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < ADJ_SLOTS) {
        double tsum = 0.0;
        if (threadIdx.x == 0)
            for (int wi = 0; wi < 8; ++wi) tsum += red[wi];
        partials[(size_t)blockIdx.x * ADJ_SLOTS + threadIdx.x] = tsum;
    }
}

// Sum of the per-block partials in a fixed order.
__global__ void __launch_bounds__(256) k_adjoint_reduce(const double* partials, uint32_t blocks, double* out) {
    __shared__ double red[256];
    for (int k = 0; k < ADJ_SLOTS; ++k) {
        double s = 0.0;
        for (uint32_t b = threadIdx.x; b < blocks; b += blockDim.x) s += partials[(size_t)b * ADJ_SLOTS + k];
        red[threadIdx.x] = s;
        __syncthreads();
        for (uint32_t st = blockDim.x / 2; st > 0; st >>= 1) {
            if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[k] = red[0];
        __syncthreads();
    }
}

}  // namespace srk
