// Binned star footprints for the batched fast path (star_light, star.rs:240-286).
//
// A star's cone event depends on the observer, not on the pixel, so it is computed once per
// (observer, star) and projected onto the image. Its footprint only reaches pixels whose direction
// is within atan(2.4 * spread) of the star's (the 4-sigma cut of star.rs:266-270, spread <= the
// pixel pitch), so each star is listed in the 16x16 tiles a generous radius around its projection
// covers (count, prefix sum, fill: compact lists of any length). A tile then sorts its list by star
// index in shared memory and every pixel sums star_term over it in that order: the stars it skips
// are exactly stars whose term the cut rejects, so the sum is the brute force sum bit for bit.
// A tile whose list does not fit (longer than STAR_SORT_CAP, or past the list buffer) sums every
// star instead. Observers outside the binning's assumptions (stars_binned_for in
// sr_kernels.h) keep the brute force in the shading kernel. Included by sr_fast.cu, which defines
// find_obs, cam_of and ObsDev.
#pragma once

namespace srk {

constexpr uint32_t STAR_SORT_CAP = 8192;  // entries a tile sorts in shared memory (32 KB)

struct StarBinArgs {
    const SrGpuUniforms* U;
    const float4* cam;
    const ObsDev* obs;
    const float4* stars;  // headers then segments
    uint32_t n, num_stars;
    float4* cd;           // per (observer, star): cone event offset and 4-velocity
    float4* cu;
    uint4* rect;          // per (observer, star): tiles x0, x1, y0, y1 (x0 > x1: none)
    uint32_t* count;      // per star tile: listed stars
    const uint32_t* offset;  // per star tile: start of its list (exclusive prefix sum of count)
    uint32_t* fill;       // per star tile: entries written so far
    uint32_t* list;
    uint32_t list_cap;
};

// Pass 1: the cone event of (observer, star), its footprint's tile rectangle, and the tile counts.
__global__ void __launch_bounds__(256) k_star_bin(StarBinArgs a) {
    const uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= (uint64_t)a.n * a.num_stars) return;
    const uint32_t o = (uint32_t)(gi / a.num_stars), i = (uint32_t)(gi % a.num_stars);
    a.rect[gi] = make_uint4(1u, 0u, 1u, 0u);
    const SrGpuUniforms& U = a.U[o];
    if (!stars_binned_for(U, a.num_stars)) return;
    const Cam cam = cam_of(a.cam, o);
    float4 ro, rd;
    float sx, sy;
    camera_ray(U, cam, 0, 0, &ro, &rd, &sx, &sy);  // the ray origin is the same for every pixel
    const float cone = U.slice_mode == 0u ? -1.0f : (U.slice_mode == 2u ? 1.0f : 0.0f);
    const float4 hd = __ldg(a.stars + i);
    float4 cd, cu;
    if (!cone_event(a.stars + a.num_stars, __float_as_uint(hd.z), __float_as_uint(hd.w), ro, cam.e0, cone, &cd, &cu))
        return;
    a.cd[gi] = cd;
    a.cu[gi] = cu;
    // The star's direction in the camera frame.
    const float tau = -mdot(cd, cam.e0);
    const float4 r = add4(cd, mul4(cam.e0, -tau));
    const float r1 = mdot(r, cam.e1), r2 = mdot(r, cam.e2), r3 = mdot(r, cam.e3);
    const float rn = sqrtf(r1 * r1 + r2 * r2 + r3 * r3);
    if (!(rn > 0.0f)) return;
    const float W = (float)U.size[0], H = (float)U.size[1];
    const float hw = U.half_wh[0], hh = U.half_wh[1];
    // Angles from the view axis: the star's alpha; the pixels' at most amax; the footprint's theta.
    const float alpha = acosf(fminf(fmaxf(r3 / rn, -1.0f), 1.0f));
    const float amax = atanf(sqrtf(hw * hw + hh * hh));
    const float theta = 2.4f * (2.0f * hh / H) * 1.1f + 1e-4f;
    if (alpha - theta > amax + 0.01f) return;  // no pixel direction comes within theta of the star
    const float ssx = r1 / r3, ssy = r2 / r3;
    // Radius in the tangent plane (the radial stretch is the worst case), then in pixels.
    const float rt = (tanf(alpha + theta) - tanf(alpha)) * 1.25f;
    const float rpx = rt / (2.0f * hw / W) + 2.0f, rpy = rt / (2.0f * hh / H) + 2.0f;
    const float cx = (ssx / hw + 1.0f) * 0.5f * W - 0.5f, cy = (1.0f - ssy / hh) * 0.5f * H - 0.5f;
    if (!(cx + rpx >= 0.0f && cx - rpx <= W - 1.0f && cy + rpy >= 0.0f && cy - rpy <= H - 1.0f)) return;
    const ObsDev& od = a.obs[o];
    const uint32_t tx16 = (od.width + STAR_TILE - 1) / STAR_TILE, ty16 = (od.height + STAR_TILE - 1) / STAR_TILE;
    const int tx0 = max(0, (int)floorf((cx - rpx) / STAR_TILE)), tx1 = min((int)tx16 - 1, (int)floorf((cx + rpx) / STAR_TILE));
    const int ty0 = max(0, (int)floorf((cy - rpy) / STAR_TILE)), ty1 = min((int)ty16 - 1, (int)floorf((cy + rpy) / STAR_TILE));
    if (tx0 > tx1 || ty0 > ty1) return;
    a.rect[gi] = make_uint4((uint32_t)tx0, (uint32_t)tx1, (uint32_t)ty0, (uint32_t)ty1);
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) atomicAdd(a.count + od.star_tile_base + (uint32_t)ty * tx16 + (uint32_t)tx, 1u);
}

// Pass 2: each (observer, star) writes its index into the lists of its tiles.
__global__ void __launch_bounds__(256) k_star_fill(StarBinArgs a) {
    const uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= (uint64_t)a.n * a.num_stars) return;
    const uint4 rc = a.rect[gi];
    if (rc.x > rc.y) return;
    const uint32_t o = (uint32_t)(gi / a.num_stars), i = (uint32_t)(gi % a.num_stars);
    const ObsDev& od = a.obs[o];
    const uint32_t tx16 = (od.width + STAR_TILE - 1) / STAR_TILE;
    for (uint32_t ty = rc.z; ty <= rc.w; ++ty)
        for (uint32_t tx = rc.x; tx <= rc.y; ++tx) {
            const uint32_t tile = od.star_tile_base + ty * tx16 + tx;
            const uint64_t k = (uint64_t)__ldg(a.offset + tile) + atomicAdd(a.fill + tile, 1u);
            if (k < a.list_cap) a.list[k] = i;
        }
}

struct StarTileArgs {
    SceneDev s;
    const SrGpuUniforms* U;
    const float4* cam;
    const ObsDev* obs;
    const uint32_t* star_pre;  // star-tile prefix over observers (n + 1)
    uint32_t n;
    const float4* hits;
    const uint32_t* slots;
    const float4* cd;
    const float4* cu;
    const uint32_t* count;
    const uint32_t* offset;
    const uint32_t* list;
    uint32_t list_cap;
    float4* hdr;
    BBConst bb;
};

// One 16x16 tile per block: sort the tile's stars by index, then every pixel adds its star sum to
// the HDR colour the shading kernel wrote (the same `colour + stars` addition as the shading).
__global__ void __launch_bounds__(256) k_star_tiles(StarTileArgs a) {
    extern __shared__ uint32_t keys[];  // STAR_SORT_CAP entries
    const uint32_t tile = blockIdx.x;
    const uint32_t o = find_obs(a.star_pre, a.n, tile);
    const SrGpuUniforms& U = a.U[o];
    if (!stars_binned_for(U, a.s.num_stars)) return;  // uniform over the block
    const ObsDev& od = a.obs[o];
    const uint32_t local = tile - __ldg(a.star_pre + o);
    const uint32_t tx16 = (od.width + STAR_TILE - 1) / STAR_TILE;
    const uint32_t px = (local % tx16) * STAR_TILE + threadIdx.x % STAR_TILE;
    const uint32_t py = (local / tx16) * STAR_TILE + threadIdx.x / STAR_TILE;
    const bool inside = px < od.width && py < od.height;
    __shared__ int bad;
    const uint32_t cnt = a.count[tile], off = a.offset[tile];
    bool brute = cnt > STAR_SORT_CAP || (uint64_t)off + cnt > a.list_cap;
    if (!brute) {
        uint32_t p2 = 1;
        while (p2 < cnt) p2 <<= 1;
        if (threadIdx.x == 0) bad = 0;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) {
            const uint32_t v = k < cnt ? a.list[off + k] : 0xFFFFFFFFu;
            if (k < cnt && v >= a.s.num_stars) bad = 1;  // a list this pass did not fill: sum every star
            keys[k] = v;
        }
        __syncthreads();
        brute = bad != 0;
    }
    if (!brute) {
        uint32_t p2 = 1;
        while (p2 < cnt) p2 <<= 1;
        // Bitonic sort of keys[0, p2) (p2 <= STAR_SORT_CAP), ascending.
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
    if (!inside) return;
    const Cam cam = cam_of(a.cam, o);
    float4 ro, rd;
    float sx, sy;
    camera_ray(U, cam, px, py, &ro, &rd, &sx, &sy);
    const uint32_t l = py * od.width + px, p = od.pix_base + l;
    const uint32_t slot = a.slots[p];
    const float lambda_max = slot != 0xFFFFFFFFu ? a.hits[p].x : INFINITY;
    F3 total;
    if (brute) {
        total = stars_brute(a.s, U, cam, ro, rd, sx, sy, lambda_max, a.bb);
    } else {
        float4 n;
        float spread, cone;
        star_ray(U, cam, rd, sx, sy, &n, &spread, &cone);
        const BB bb{a.bb.r5, a.bb.g5, a.bb.b5, a.bb.wr, a.bb.wg, a.bb.wb};
        total = F3{0.0f, 0.0f, 0.0f};
        const size_t base = (size_t)o * a.s.num_stars;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t i = keys[k];
            const float4 hd = __ldg(a.s.stars + i);
            F3 c;
            if (star_term(__ldg(a.cd + base + i), __ldg(a.cu + base + i), cam.e0, cone, n, spread, lambda_max, hd.x, hd.y,
                          bb, &c))
                total = add(total, c);
        }
    }
    float4* h = a.hdr + (size_t)od.pyr_base + l;
    const float4 v = *h;
    *h = make_float4(v.x + total.x, v.y + total.y, v.z + total.z, 0.0f);
}

}  // namespace srk
