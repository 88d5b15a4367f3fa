// The fast path: the B200 node layout, and a batch of observers rendered as one sequence of
// launches (captured once into a CUDA graph and replayed):
//
//   k_camera_batch   FP64 observers (tetrad from rapidity in double, event rebased to the anchor)
//   k_trace_batch    persistent: each warp takes a 32-pixel tile of any observer from one global
//                    counter and writes the primary hit records
//   k_shade_batch    one thread per pixel: interpolation and shading; a pixel whose main-light
//                    shadow ray is due goes to a compacted queue instead (warp-aggregated append)
//   k_shadow_batch   persistent any-hit traversal of the queue, so the few long shadow rays spread
//                    over every SM instead of stretching the blocks that happen to hold them
//   k_finish_batch   the queued pixels, shaded with their shadow result
//   bloom            the pyramid of every observer, one launch per level
//
// Shading is one device function used by k_shade_batch and k_finish_batch, so a queued pixel's
// colour is computed by the same operations as any other (renderer.rs:414-489, 609-653).
#include <cub/cub.cuh>

#include <cstring>

#include "sr_camera.cuh"
#include "sr_fast.h"
#include "sr_shade.cuh"
#include "sr_traverse.cuh"

namespace srk {

using namespace srd;

// ---------------------------------------------------------------------------------------------
// Layout build.
// ---------------------------------------------------------------------------------------------
__global__ void k_wide_flags(const SrGpuNode* nodes, uint32_t n, uint32_t* flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = nodes[i].count == 0 ? 1u : 0u;
}

__global__ void k_wide_fill(const SrGpuNode* nodes, uint32_t n, const uint32_t* wid, float4* boxes, uint2* refs) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nodes[i].count != 0) return;
    const SrGpuNode& nd = nodes[i];
    uint32_t c[2] = {nd.left, nd.right_or_first}, ref[2];
    float4* b = boxes + 4ull * wid[i];
    for (int k = 0; k < 2; ++k) {
        const SrGpuNode& ch = nodes[c[k]];
        b[2 * k] = make_float4(ch.min[0], ch.min[1], ch.min[2], ch.min[3]);
        b[2 * k + 1] = make_float4(ch.max[0], ch.max[1], ch.max[2], ch.max[3]);
        ref[k] = ch.count > 0 ? pack_leaf(ch.right_or_first, ch.count) : wid[c[k]];
    }
    refs[wid[i]] = make_uint2(ref[0], ref[1]);
}

cudaError_t fast_init(FastCtx& c, const cudaDeviceProp& prop) {
    c.num_sms = prop.multiProcessorCount;
    c.max_smem = (int)prop.sharedMemPerBlockOptin;
    return cudaSuccess;
}

void fast_release(FastCtx& c) {
    for (auto& kv : c.graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    c.graphs.clear();
}

cudaError_t fast_build(FastCtx& c, FastScene& s, const SrGpuNode* nodes, uint32_t n, uint32_t depth, uint32_t num_prims,
                       uint32_t max_leaf, cudaStream_t st) {
    (void)c;
    s.num_wide = 0;
    s.depth = depth;
    s.empty = n == 0;
    s.usable = depth <= FAST_MAX_DEPTH && num_prims < MAX_PACKED_PRIMS && max_leaf <= MAX_LEAF_PRIMS;
    if (n == 0 || !s.usable) return cudaSuccess;
    SrGpuNode root;
    cudaError_t e = cudaMemcpyAsync(&root, nodes, sizeof(root), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int k = 0; k < 4; ++k) { s.root_min[k] = root.min[k]; s.root_max[k] = root.max[k]; }
    if (root.count > 0) {
        s.root_ref = pack_leaf(root.right_or_first, root.count);
        return cudaSuccess;
    }
    s.root_ref = 0;  // internal root: wide node 0 (depth-first order)
    size_t temp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, st);
    if ((e = s.scratch.ensure(2 * (size_t)n * 4 + temp + 512)) != cudaSuccess) return e;
    uint32_t* flags = s.scratch.as<uint32_t>();
    uint32_t* wid = flags + n;
    uintptr_t tp = reinterpret_cast<uintptr_t>(wid + n);
    void* tmp = reinterpret_cast<void*>((tp + 255) & ~uintptr_t(255));
    k_wide_flags<<<(n + 255) / 256, 256, 0, st>>>(nodes, n, flags);
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, temp, flags, wid, (int)n, st)) != cudaSuccess) return e;
    uint32_t last[2] = {0, 0};
    cudaMemcpyAsync(&last[0], wid + n - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last[1], flags + n - 1, 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    s.num_wide = last[0] + last[1];
    if ((e = s.boxes.ensure((size_t)s.num_wide * 64)) != cudaSuccess) return e;
    if ((e = s.refs.ensure((size_t)s.num_wide * 8)) != cudaSuccess) return e;
    k_wide_fill<<<(n + 255) / 256, 256, 0, st>>>(nodes, n, wid, s.boxes.as<float4>(), s.refs.as<uint2>());
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    s.scratch.ensure(0);
    return e;
}

SrTuning fast_default_tuning(const FastCtx& c) {
    (void)c;
    SrTuning t{};
    t.block_threads = 128;
    t.blocks_per_sm = 8;
    t.stack_depth = FAST_STACK;
    t.smem_levels = 0;
    t.tile_w = 8;
    t.tile_h = 4;
    return t;
}

bool fast_tuning_valid(const FastCtx& c, const SrTuning& t) {
    (void)c;
    bool bt = t.block_threads == 64 || t.block_threads == 128 || t.block_threads == 256 || t.block_threads == 512;
    return bt && t.blocks_per_sm >= 1 && t.blocks_per_sm <= 16 && t.tile_w >= 1 && t.tile_w * t.tile_h == 32 &&
           t.stack_depth == (uint32_t)FAST_STACK && t.smem_levels == 0;
}

// ---------------------------------------------------------------------------------------------
// Batch kernels.
// ---------------------------------------------------------------------------------------------

// The observer holding global index x: the largest o with pre[o] <= x (pre[0] = 0, pre[n] = total).
__device__ __forceinline__ uint32_t find_obs(const uint32_t* pre, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(pre + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ Cam cam_of(const float4* cam, uint32_t o) {
    const float4* c = cam + 6ull * o;
    Cam r;
    r.pos = __ldg(c);
    r.e0 = __ldg(c + 1);
    r.e1 = __ldg(c + 2);
    r.e2 = __ldg(c + 3);
    r.e3 = __ldg(c + 4);
    r.frontier = __ldg(c + 5);
    return r;
}

__global__ void k_camera_batch(uint32_t n, const SrGpuUniforms* U, const SrCameraF64* cam64, const ObsDev* obs,
                               double a0, double a1, double a2, double a3, float4* cam) {
    uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    float4* out = cam + 6ull * o;
    if (obs[o].has_cam64) {
        double anchor[4] = {a0, a1, a2, a3};
        camera_f64(cam64[o], anchor, U[o], out);
    } else {
        const SrGpuUniforms& u = U[o];
        out[0] = v4(u.cam_pos[0], u.cam_pos[1], u.cam_pos[2], u.cam_pos[3]);
        for (int a = 0; a < 4; ++a) out[1 + a] = v4(u.e[a][0], u.e[a][1], u.e[a][2], u.e[a][3]);
        out[5] = v4(u.frontier_origin[0], u.frontier_origin[1], u.frontier_origin[2], u.frontier_origin[3]);
    }
}

struct TraceBatchArgs {
    WideScene ws;
    const SrGpuUniforms* U;
    const float4* cam;
    const ObsDev* obs;
    const uint32_t* tile_pre;
    uint32_t n, total_tiles, tile_w, tile_h;
    float4* hits;
    uint32_t* slots;
    uint32_t* counter;
    uint32_t* err;
    unsigned long long* work;
};

__device__ __forceinline__ void add_work(unsigned long long* c, const Work& w) {
    atomicAdd(c + 0, (unsigned long long)w.nodes);
    atomicAdd(c + 1, (unsigned long long)w.leaves);
    atomicAdd(c + 2, (unsigned long long)w.tets);
}

template <bool COUNT>
__global__ void __launch_bounds__(512) k_trace_batch(TraceBatchArgs a) {
    const uint32_t lane = threadIdx.x & 31u;
    Work work{0, 0, 0};
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(a.counter, 1u);
        t = __shfl_sync(0xFFFFFFFFu, t, 0);
        if (t >= a.total_tiles) break;
        uint32_t o = find_obs(a.tile_pre, a.n, t);
        const ObsDev& od = a.obs[o];
        uint32_t lt = t - __ldg(a.tile_pre + o);
        uint32_t tiles_x = od.tiles_x;
        uint32_t px = (lt % tiles_x) * a.tile_w + lane % a.tile_w;
        uint32_t py = (lt / tiles_x) * a.tile_h + lane / a.tile_w;
        uint32_t w = od.width, h = od.height;
        if (px >= w || py >= h) continue;
        const Cam cam = cam_of(a.cam, o);
        float4 ro, rd;
        float sx, sy;
        camera_ray(a.U[o], cam, px, py, &ro, &rd, &sx, &sy);
        GeomHit gh;
        int slot = trace_wide<COUNT>(a.ws, ro, rd, 1e-3f, 180.0f, &gh, a.err, &work);
        size_t p = (size_t)od.pix_base + (size_t)py * w + px;
        a.hits[p] = make_float4(gh.lambda, gh.u, gh.v, gh.w);
        a.slots[p] = slot < 0 ? 0xFFFFFFFFu : (uint32_t)slot;
    }
    if (COUNT) add_work(a.work, work);
}

struct ShadeBatchArgs {
    SceneDev s;
    WideScene ws;
    const SrGpuUniforms* U;
    const float4* cam;
    const ObsDev* obs;
    const uint32_t* pix_pre;
    uint32_t n, total_px;
    const float4* hits;
    const uint32_t* slots;
    float4* hdr;
    uint32_t* hit_id;
    float* lambda;
    float* tau;
    ShadowRay* queue;
    uint8_t* qflags;
    uint32_t* counters;  // [0] shadow rays, [1] errors, [2] tile counter, [3] queue length
    unsigned long long* work;
    BBConst bb;
};

// Any-hit queries from inside the shading, traced on the spot (the flash rays of a pixel).
template <bool COUNT>
struct InlineOccluder {
    const WideScene* s;
    uint32_t* err;
    Work* work;
    __device__ bool operator()(float4 o, float4 d, float t0, float t1) { return occluded_wide<COUNT>(*s, o, d, t0, t1, err, work); }
};
// The main light's shadow ray of a queued pixel, already traced.
struct QueuedOccluder {
    bool result;
    __device__ bool operator()(float4, float4, float, float) const { return result; }
};

struct PixelRef {
    uint32_t o, px, py, l;
};
__device__ __forceinline__ PixelRef pixel_of(const ShadeBatchArgs& a, uint32_t p) {
    PixelRef r;
    r.o = find_obs(a.pix_pre, a.n, p);
    r.l = p - __ldg(a.pix_pre + r.o);
    uint32_t w = a.obs[r.o].width;
    r.px = r.l % w;
    r.py = r.l / w;
    return r;
}

// The HDR colour of pixel `p` (renderer.rs:369-404), with shadow rays answered by `occ`.
template <class Occ>
__device__ __forceinline__ F3 pixel_color(const ShadeBatchArgs& a, const PixelRef& pr, uint32_t p, Occ& occ, Hit* h,
                                          uint32_t* shadow_rays) {
    const SrGpuUniforms& U = a.U[pr.o];
    const Cam cam = cam_of(a.cam, pr.o);
    float4 ro, rd;
    float sx, sy;
    camera_ray(U, cam, pr.px, pr.py, &ro, &rd, &sx, &sy);
    uint32_t slot = a.slots[p];
    F3 color;
    if (slot != 0xFFFFFFFFu) {
        float4 hr = a.hits[p];
        GeomHit gh{hr.x, hr.y, hr.z, hr.w};
        interpolate(a.s.attrs + 12u * slot, ro, rd, gh, h);
        color = shade_hit(a.s, U, cam, rd, *h, occ, shadow_rays);
        if (U.num_haze > 0u) color = apply_haze(color, h->event, U);
    } else {
        color = shade_sky(rd);
    }
    if (U.mode == 0u && a.s.num_stars > 0u)
        color = add(color, stars_brute(a.s, U, cam, ro, rd, sx, sy, slot != 0xFFFFFFFFu ? h->lambda : INFINITY, a.bb));
    return color;
}

__device__ __forceinline__ void write_pixel(const ShadeBatchArgs& a, const PixelRef& pr, uint32_t p, F3 color, const Hit& h,
                                            uint32_t slot) {
    const ObsDev& od = a.obs[pr.o];
    a.hdr[(size_t)od.pyr_base + pr.l] = make_float4(color.x, color.y, color.z, 0.0f);
    if (a.hit_id)
        a.hit_id[p] = slot == 0xFFFFFFFFu ? 0xFFFFFFFFu : (a.s.leaf_to_orig ? __ldg(a.s.leaf_to_orig + slot) : slot);
    if (a.lambda) a.lambda[p] = slot == 0xFFFFFFFFu ? 0.0f : h.lambda;
    if (a.tau) a.tau[p] = slot == 0xFFFFFFFFu ? 0.0f : h.tau;
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_shade_batch(ShadeBatchArgs a) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = p < a.total_px;
    // Does this pixel's main light need a shadow ray (compute_illumination, renderer.rs:617-645)?
    bool queued = false;
    ShadowRay sr;
    PixelRef pr{0, 0, 0, 0};
    uint32_t slot = 0xFFFFFFFFu;
    if (live) {
        pr = pixel_of(a, p);
        slot = a.slots[p];
        const SrGpuUniforms& U = a.U[pr.o];
        if (slot != 0xFFFFFFFFu && U.mode == 0u && U.shadow_mode != 0u && U.num_flashes == 0u) {
            const Cam cam = cam_of(a.cam, pr.o);
            float4 ro, rd;
            float sx, sy;
            camera_ray(U, cam, pr.px, pr.py, &ro, &rd, &sx, &sy);
            float4 hr = a.hits[p];
            GeomHit gh{hr.x, hr.y, hr.z, hr.w};
            Hit h;
            interpolate(a.s.attrs + 12u * slot, ro, rd, gh, &h);
            Mat m = load_mat(a.s.mats, h.material);
            if (m.pattern == 0u) {
                float4 tl;
                float dist;
                light_ray(U, cam, h.event, &tl, &dist);
                if (fmaxf(rest_frame_cos(tl, h.normal, h.four_vel), 0.0f) > 0.0f) {
                    queued = true;
                    sr.origin = h.event;
                    sr.dir = tl;
                    sr.t_max = dist - 2e-3f;
                    sr.pixel = p;
                }
            }
        }
    }
    // Warp-aggregated append to the shadow queue.
    unsigned mask = __ballot_sync(0xFFFFFFFFu, queued);
    if (mask) {
        uint32_t lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u, base = 0;
        if (lane == leader) base = atomicAdd(a.counters + 3, (uint32_t)__popc(mask));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (queued) a.queue[base + __popc(mask & ((1u << lane) - 1u))] = sr;
    }
    if (!live || queued) return;
    Work work{0, 0, 0};
    InlineOccluder<COUNT> occ{&a.ws, a.counters + 1, &work};
    uint32_t shadow_rays = 0;
    Hit h;
    h.lambda = 0.0f;
    h.tau = 0.0f;
    F3 color = pixel_color(a, pr, p, occ, &h, &shadow_rays);
    write_pixel(a, pr, p, color, h, slot);
    if (shadow_rays) atomicAdd(a.counters, shadow_rays);
    if (COUNT && work.nodes) add_work(a.work + 3, work);
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_shadow_batch(WideScene ws, const ShadowRay* queue, const uint32_t* qlen,
                                                       uint8_t* qflags, uint32_t* fetch, uint32_t* err,
                                                       unsigned long long* work_out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = *qlen;
    Work work{0, 0, 0};
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(fetch, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= n) break;
        uint32_t i = base + lane;
        if (i < n) {
            const ShadowRay& r = queue[i];
            qflags[i] = occluded_wide<COUNT>(ws, r.origin, r.dir, 2e-3f, r.t_max, err, &work) ? 1 : 0;
        }
    }
    if (COUNT && work.nodes) add_work(work_out + 3, work);
}

__global__ void __launch_bounds__(256) k_finish_batch(ShadeBatchArgs a) {
    const uint32_t n = a.counters[3];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t p = a.queue[i].pixel;
        PixelRef pr = pixel_of(a, p);
        QueuedOccluder occ{a.qflags[i] != 0};
        uint32_t shadow_rays = 0;
        Hit h;
        F3 color = pixel_color(a, pr, p, occ, &h, &shadow_rays);
        write_pixel(a, pr, p, color, h, a.slots[p]);
        atomicAdd(a.counters, shadow_rays);
    }
}

// Bloom over every observer's pyramid (bloom.rs:54-125); `pre` is the per-observer prefix of the
// level's pixel counts.
__constant__ float DOWN_WB[4] = {0.125f, 0.375f, 0.375f, 0.125f};

__global__ void k_bloom_down_batch(float4* hdr, const ObsDev* obs, const uint32_t* pre, uint32_t n, int k) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= __ldg(pre + n)) return;
    uint32_t o = find_obs(pre, n, i);
    const ObsDev& od = obs[o];
    uint32_t l = i - __ldg(pre + o);
    uint32_t dw = od.lw[k], x = l % dw, y = l / dw;
    uint32_t sw = od.lw[k - 1], sh = od.lh[k - 1];
    const float4* src = hdr + od.pyr_base + od.loff[k - 1];
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int syi = 2 * (int)y - 1 + j;
        syi = syi < 0 ? 0 : (syi > (int)sh - 1 ? (int)sh - 1 : syi);
        float rx = 0.0f, ry = 0.0f, rz = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int sxi = 2 * (int)x - 1 + q;
            sxi = sxi < 0 ? 0 : (sxi > (int)sw - 1 ? (int)sw - 1 : sxi);
            float4 v = src[(size_t)syi * sw + sxi];
            rx = rx + v.x * DOWN_WB[q];
            ry = ry + v.y * DOWN_WB[q];
            rz = rz + v.z * DOWN_WB[q];
        }
        ax = ax + rx * DOWN_WB[j];
        ay = ay + ry * DOWN_WB[j];
        az = az + rz * DOWN_WB[j];
    }
    hdr[od.pyr_base + od.loff[k] + l] = make_float4(ax, ay, az, 0.0f);
}

__device__ __forceinline__ float4 upsample_b(const float4* c, uint32_t cw, uint32_t ch, uint32_t x, uint32_t y) {
    uint32_t mx = x / 2, my = y / 2;
    int ox = (x % 2 == 0) ? (int)mx - 1 : (int)mx + 1;
    int oy = (y % 2 == 0) ? (int)my - 1 : (int)my + 1;
    uint32_t x1 = (uint32_t)(ox < 0 ? 0 : (ox > (int)cw - 1 ? (int)cw - 1 : ox));
    uint32_t y1 = (uint32_t)(oy < 0 ? 0 : (oy > (int)ch - 1 ? (int)ch - 1 : oy));
    float4 A = c[(size_t)my * cw + mx], B = c[(size_t)my * cw + x1];
    float4 E = c[(size_t)y1 * cw + mx], G = c[(size_t)y1 * cw + x1];
    float r0x = A.x * 0.75f + B.x * 0.25f, r0y = A.y * 0.75f + B.y * 0.25f, r0z = A.z * 0.75f + B.z * 0.25f;
    float r1x = E.x * 0.75f + G.x * 0.25f, r1y = E.y * 0.75f + G.y * 0.25f, r1z = E.z * 0.75f + G.z * 0.25f;
    return make_float4(r0x * 0.75f + r1x * 0.25f, r0y * 0.75f + r1y * 0.25f, r0z * 0.75f + r1z * 0.25f, 0.0f);
}

__global__ void k_bloom_up_batch(float4* hdr, const ObsDev* obs, const uint32_t* pre, uint32_t n, int k) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= __ldg(pre + n)) return;
    uint32_t o = find_obs(pre, n, i);
    const ObsDev& od = obs[o];
    uint32_t l = i - __ldg(pre + o);
    uint32_t w = od.lw[k], x = l % w, y = l / w;
    float4 up = upsample_b(hdr + od.pyr_base + od.loff[k + 1], od.lw[k + 1], od.lh[k + 1], x, y);
    float4* dst = hdr + od.pyr_base + od.loff[k] + l;
    float4 v = *dst;
    *dst = make_float4(v.x + up.x, v.y + up.y, v.z + up.z, 0.0f);
}

__global__ void __launch_bounds__(256) k_bloom_composite_batch(const float4* hdr, const ObsDev* obs, const uint32_t* pre,
                                                               uint32_t n, uint32_t* rgb, const uint32_t* tables) {
    __shared__ uint8_t lut[SR_GAMMA_LUT_SIZE];
    for (uint32_t i = threadIdx.x; i < SR_GAMMA_LUT_SIZE; i += blockDim.x) lut[i] = (uint8_t)__ldg(tables + i);
    __syncthreads();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= __ldg(pre + n)) return;
    uint32_t o = find_obs(pre, n, i);
    const ObsDev& od = obs[o];
    uint32_t l = i - __ldg(pre + o);
    uint32_t w = od.lw[0], x = l % w, y = l / w;
    const float strength = 0.04f;
    const float keep = 1.0f - strength;
    const float halo = strength / (float)SR_BLOOM_LEVELS;
    float4 up = upsample_b(hdr + od.pyr_base + od.loff[1], od.lw[1], od.lh[1], x, y);
    float4 c = hdr[od.pyr_base + l];
    float cx = c.x * keep + up.x * halo, cy = c.y * keep + up.y * halo, cz = c.z * keep + up.z * halo;
    float mx = cx / (1.0f + cx * 0.35f), my = cy / (1.0f + cy * 0.35f), mz = cz / (1.0f + cz * 0.35f);
    mx = mx < 0.0f ? 0.0f : (mx > 1.0f ? 1.0f : mx);
    my = my < 0.0f ? 0.0f : (my > 1.0f ? 1.0f : my);
    mz = mz < 0.0f ? 0.0f : (mz > 1.0f ? 1.0f : mz);
    const float scale = (float)(SR_GAMMA_LUT_SIZE - 1);
    float fx = mx * scale, fy = my * scale, fz = mz * scale;
    uint32_t ix = fx > 0.0f ? (uint32_t)fx : 0u, iy = fy > 0.0f ? (uint32_t)fy : 0u, iz = fz > 0.0f ? (uint32_t)fz : 0u;
    rgb[i] = ((uint32_t)lut[ix] << 16) | ((uint32_t)lut[iy] << 8) | (uint32_t)lut[iz];
}

// ---------------------------------------------------------------------------------------------
// The batch sequence.
// ---------------------------------------------------------------------------------------------
namespace {

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

struct Shape {
    uint32_t n = 0, total_tiles = 0, total_px = 0, total_pyr = 0;
    std::vector<ObsDev> obs;
    std::vector<uint32_t> pre;  // (SR_BLOOM_LEVELS + 2) rows of n + 1: tiles, then levels 0..6
};

Shape make_shape(const BatchRequest& r, const SrTuning& t) {
    Shape s;
    s.n = r.n;
    s.obs.resize(r.n);
    const uint32_t rows = SR_BLOOM_LEVELS + 2, stride = r.n + 1;
    s.pre.assign((size_t)rows * stride, 0);
    uint32_t tiles = 0, px = 0, pyr = 0;
    for (uint32_t i = 0; i < r.n; ++i) {
        ObsDev& o = s.obs[i];
        std::memset(&o, 0, sizeof(o));
        o.width = r.u[i].size[0];
        o.height = r.u[i].size[1];
        o.tiles_x = (o.width + t.tile_w - 1) / t.tile_w;
        o.tile_base = tiles;
        o.pix_base = px;
        o.pyr_base = pyr;
        o.has_cam64 = r.cam64 ? 1u : 0u;
        Pyramid p = make_pyramid(o.width, o.height);
        for (int k = 0; k <= SR_BLOOM_LEVELS; ++k) { o.lw[k] = p.w[k]; o.lh[k] = p.h[k]; o.loff[k] = p.off[k]; }
        o.loff[SR_BLOOM_LEVELS + 1] = p.off[SR_BLOOM_LEVELS + 1];
        s.pre[0 * stride + i] = tiles;
        for (int k = 0; k <= SR_BLOOM_LEVELS; ++k) {
            uint32_t* row = &s.pre[(size_t)(1 + k) * stride];
            row[i + 1] = row[i] + p.w[k] * p.h[k];
        }
        tiles += o.tiles_x * ((o.height + t.tile_h - 1) / t.tile_h);
        px += o.width * o.height;
        pyr += p.off[SR_BLOOM_LEVELS + 1];
    }
    s.pre[r.n] = tiles;
    s.total_tiles = tiles;
    s.total_px = px;
    s.total_pyr = pyr;
    return s;
}

}  // namespace

float4* fast_batch_hdr(FastCtx& c, uint32_t pyr_base) { return c.hdr.as<float4>() + pyr_base; }

cudaError_t fast_render_batch(FastCtx& c, const FastScene& s, const SrTuning& t, const SceneDev& sd,
                              const double anchor[4], const BBConst& bb, uint32_t* counters, const BatchRequest& r,
                              cudaStream_t st) {
    if (r.n == 0) return cudaSuccess;
    Shape sh = make_shape(r, t);
    const uint32_t n = r.n, stride = n + 1;
    cudaError_t e;
    // Buffers (grown on demand; a growth invalidates every captured graph).
    size_t old_hits = c.hits.bytes, old_hdr = c.hdr.bytes, old_U = c.U.bytes, old_q = c.queue.bytes, old_rgb = c.rgb.bytes;
    if ((e = c.U.ensure(n * sizeof(SrGpuUniforms))) != cudaSuccess) return e;
    if ((e = c.cam64.ensure(n * sizeof(SrCameraF64))) != cudaSuccess) return e;
    if ((e = c.cam.ensure(n * 6 * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.obs.ensure(n * sizeof(ObsDev))) != cudaSuccess) return e;
    if ((e = c.lvl_pre.ensure(sh.pre.size() * 4)) != cudaSuccess) return e;
    if ((e = c.hits.ensure((size_t)sh.total_px * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.slots.ensure((size_t)sh.total_px * 4)) != cudaSuccess) return e;
    if ((e = c.queue.ensure((size_t)sh.total_px * sizeof(ShadowRay))) != cudaSuccess) return e;
    if ((e = c.qflags.ensure((size_t)sh.total_px)) != cudaSuccess) return e;
    if ((e = c.hdr.ensure((size_t)sh.total_pyr * sizeof(float4))) != cudaSuccess) return e;
    if (!r.rgb && (e = c.rgb.ensure((size_t)sh.total_px * 4)) != cudaSuccess) return e;
    if ((e = c.hU.ensure(n * sizeof(SrGpuUniforms))) != cudaSuccess) return e;
    if ((e = c.hcam64.ensure(n * sizeof(SrCameraF64))) != cudaSuccess) return e;
    if ((e = c.hobs.ensure(n * sizeof(ObsDev))) != cudaSuccess) return e;
    if ((e = c.hlvl.ensure(sh.pre.size() * 4)) != cudaSuccess) return e;
    if (c.hits.bytes != old_hits || c.hdr.bytes != old_hdr || c.U.bytes != old_U || c.queue.bytes != old_q ||
        c.rgb.bytes != old_rgb)
        fast_release(c);
    // The previous batch's copies from the pinned staging must have run before it is rewritten.
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    std::memcpy(c.hU.p, r.u, n * sizeof(SrGpuUniforms));
    if (r.cam64) std::memcpy(c.hcam64.p, r.cam64, n * sizeof(SrCameraF64));
    std::memcpy(c.hobs.p, sh.obs.data(), n * sizeof(ObsDev));
    std::memcpy(c.hlvl.p, sh.pre.data(), sh.pre.size() * 4);

    uint32_t* rgb = r.rgb ? r.rgb : c.rgb.as<uint32_t>();
    WideScene ws;
    ws.boxes = s.boxes.as<float4>();
    ws.refs = s.refs.as<uint2>();
    ws.geoms = sd.geoms;
    ws.root_min = make_float4(s.root_min[0], s.root_min[1], s.root_min[2], s.root_min[3]);
    ws.root_max = make_float4(s.root_max[0], s.root_max[1], s.root_max[2], s.root_max[3]);
    ws.root_ref = s.root_ref;
    ws.empty = s.empty ? 1u : 0u;
    unsigned long long* work = reinterpret_cast<unsigned long long*>(counters + 4);
    const uint32_t* tile_pre = c.lvl_pre.as<uint32_t>();
    const uint32_t* pix_pre = tile_pre + stride;

    auto sequence = [&](bool timed) -> cudaError_t {
        cudaError_t x;
        if ((x = cudaMemcpyAsync(c.U.p, c.hU.p, n * sizeof(SrGpuUniforms), cudaMemcpyHostToDevice, st)) != cudaSuccess) return x;
        if (r.cam64 && (x = cudaMemcpyAsync(c.cam64.p, c.hcam64.p, n * sizeof(SrCameraF64), cudaMemcpyHostToDevice, st)) != cudaSuccess) return x;
        if ((x = cudaMemcpyAsync(c.obs.p, c.hobs.p, n * sizeof(ObsDev), cudaMemcpyHostToDevice, st)) != cudaSuccess) return x;
        if ((x = cudaMemcpyAsync(c.lvl_pre.p, c.hlvl.p, sh.pre.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return x;
        if ((x = cudaMemsetAsync(counters, 0, r.count_work ? 64 : 16, st)) != cudaSuccess) return x;
        k_camera_batch<<<(n + 63) / 64, 64, 0, st>>>(n, c.U.as<SrGpuUniforms>(), c.cam64.as<SrCameraF64>(), c.obs.as<ObsDev>(),
                                                     anchor[0], anchor[1], anchor[2], anchor[3], c.cam.as<float4>());
        if (timed) cudaEventRecord(r.ev[0], st);
        TraceBatchArgs ta;
        ta.ws = ws;
        ta.U = c.U.as<SrGpuUniforms>();
        ta.cam = c.cam.as<float4>();
        ta.obs = c.obs.as<ObsDev>();
        ta.tile_pre = tile_pre;
        ta.n = n;
        ta.total_tiles = sh.total_tiles;
        ta.tile_w = t.tile_w;
        ta.tile_h = t.tile_h;
        ta.hits = c.hits.as<float4>();
        ta.slots = c.slots.as<uint32_t>();
        ta.counter = counters + 2;
        ta.err = counters + 1;
        ta.work = work;
        uint32_t blocks = (uint32_t)c.num_sms * t.blocks_per_sm;
        uint32_t need = (uint32_t)(((uint64_t)sh.total_tiles * 32 + t.block_threads - 1) / t.block_threads);
        if (blocks > need) blocks = need;
        if (r.count_work) k_trace_batch<true><<<blocks, t.block_threads, 0, st>>>(ta);
        else k_trace_batch<false><<<blocks, t.block_threads, 0, st>>>(ta);
        if ((x = cudaGetLastError()) != cudaSuccess) return x;
        if (timed) cudaEventRecord(r.ev[1], st);
        ShadeBatchArgs sa;
        sa.s = sd;
        sa.ws = ws;
        sa.U = ta.U;
        sa.cam = ta.cam;
        sa.obs = ta.obs;
        sa.pix_pre = pix_pre;
        sa.n = n;
        sa.total_px = sh.total_px;
        sa.hits = ta.hits;
        sa.slots = ta.slots;
        sa.hdr = c.hdr.as<float4>();
        sa.hit_id = r.hit_id;
        sa.lambda = r.lambda;
        sa.tau = r.tau;
        sa.queue = c.queue.as<ShadowRay>();
        sa.qflags = c.qflags.as<uint8_t>();
        sa.counters = counters;
        sa.work = work;
        sa.bb = bb;
        uint32_t gpx = (sh.total_px + 255) / 256;
        if (r.count_work) k_shade_batch<true><<<gpx, 256, 0, st>>>(sa);
        else k_shade_batch<false><<<gpx, 256, 0, st>>>(sa);
        // The shadow queue: reuse the tile counter slot ([2]) for fetching after the trace is done.
        if ((x = cudaMemsetAsync(counters + 2, 0, 4, st)) != cudaSuccess) return x;
        uint32_t sblocks = (uint32_t)c.num_sms * 8;
        if (r.count_work)
            k_shadow_batch<true><<<sblocks, 256, 0, st>>>(ws, sa.queue, counters + 3, sa.qflags, counters + 2, counters + 1, work);
        else
            k_shadow_batch<false><<<sblocks, 256, 0, st>>>(ws, sa.queue, counters + 3, sa.qflags, counters + 2, counters + 1, work);
        k_finish_batch<<<(uint32_t)c.num_sms * 4, 256, 0, st>>>(sa);
        if ((x = cudaGetLastError()) != cudaSuccess) return x;
        if (timed) {
            cudaEventRecord(r.ev[2], st);
            cudaEventRecord(r.ev[3], st);
        }
        for (int k = 1; k <= SR_BLOOM_LEVELS; ++k) {
            const uint32_t* pre = tile_pre + (size_t)(1 + k) * stride;
            uint32_t tot = sh.pre[(size_t)(1 + k) * stride + n];
            k_bloom_down_batch<<<(tot + 255) / 256, 256, 0, st>>>(sa.hdr, sa.obs, pre, n, k);
        }
        for (int k = SR_BLOOM_LEVELS - 1; k >= 1; --k) {
            const uint32_t* pre = tile_pre + (size_t)(1 + k) * stride;
            uint32_t tot = sh.pre[(size_t)(1 + k) * stride + n];
            k_bloom_up_batch<<<(tot + 255) / 256, 256, 0, st>>>(sa.hdr, sa.obs, pre, n, k);
        }
        k_bloom_composite_batch<<<gpx, 256, 0, st>>>(sa.hdr, sa.obs, pix_pre, n, rgb, sd.tables);
        if ((x = cudaGetLastError()) != cudaSuccess) return x;
        if (timed) cudaEventRecord(r.ev[4], st);
        return cudaSuccess;
    };

    const bool timed = r.ev != nullptr;
    if (!r.use_graph || timed || r.count_work) return sequence(timed);

    uint64_t key = 0xC0FFEEull;
    key = mix(key, n);
    key = mix(key, r.cam64 ? 1 : 0);
    key = mix(key, reinterpret_cast<uintptr_t>(rgb));
    key = mix(key, reinterpret_cast<uintptr_t>(r.hit_id));
    key = mix(key, reinterpret_cast<uintptr_t>(r.lambda));
    key = mix(key, reinterpret_cast<uintptr_t>(r.tau));
    key = mix(key, reinterpret_cast<uintptr_t>(sd.geoms));
    key = mix(key, reinterpret_cast<uintptr_t>(ws.boxes));
    key = mix(key, ((uint64_t)t.block_threads << 32) | t.blocks_per_sm);
    key = mix(key, ((uint64_t)t.tile_w << 32) | t.tile_h);
    for (auto& o : sh.obs) key = mix(key, ((uint64_t)o.width << 32) | o.height);
    auto it = c.graphs.find(key);
    if (it == c.graphs.end()) {
        if (c.graphs.size() > 64) fast_release(c);
        GraphEntry g;
        if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return sequence(false);
        cudaError_t se = sequence(false);
        e = cudaStreamEndCapture(st, &g.graph);
        if (se != cudaSuccess || e != cudaSuccess) {
            if (g.graph) cudaGraphDestroy(g.graph);
            cudaGetLastError();
            return sequence(false);
        }
        if ((e = cudaGraphInstantiate(&g.exec, g.graph, 0)) != cudaSuccess) {
            cudaGraphDestroy(g.graph);
            cudaGetLastError();
            return sequence(false);
        }
        it = c.graphs.emplace(key, g).first;
    }
    return cudaGraphLaunch(it->second.exec, st);
}

}  // namespace srk
