// The fast path: the B200 node layout, and a batch of observers rendered as one sequence of
// launches (captured once into a CUDA graph and replayed):
//
//   k_camera_batch   FP64 observers (tetrad from rapidity in double, event rebased to the anchor)
//   k_trace_lean     persistent traversal (the default schedule): warps take 32-ray tiles from a
//                    global counter; each lane traces its pixel's primary ray (closest hit), then,
//                    when the main light needs it, the shadow ray (any hit) in the same launch.
//   k_trace_batch    the same work under the other schedules of SrTuning (per-warp chunks of
//                    tiles, partial refills, postponed or cooperative leaf tests).
//   k_shade_batch    one thread per pixel: interpolation and shading, with the main light's
//                    shadow result from the trace kernel (renderer.rs:414-489, 609-653)
//   bloom            the pyramid of every observer, one launch per level
//
// The trace kernel decides "shadow ray needed" with the same code the shading evaluates
// (checkerboard material, light in front in the surface's rest frame), and the shading checks the
// two agree.
#include <cub/cub.cuh>

#include <algorithm>
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
// The internal nodes of the top TOP_LEVELS levels, breadth first, from an internal root (node 0):
// topid[node] = its position + 1 (topid zeroed before), level_end[k] = nodes in levels 0..k. One
// thread: at most TOP_NODES nodes, once per layout build.
__global__ void k_top_levels(const SrGpuNode* nodes, uint32_t* topid, uint32_t* level_end) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t q[TOP_NODES];
    uint32_t m = 1, start = 0, end = 1;
    q[0] = 0;
    topid[0] = 1;
    level_end[0] = 1;
    for (uint32_t lv = 1; lv < TOP_LEVELS; ++lv) {
        for (uint32_t i = start; i < end; ++i) {
            const SrGpuNode& nd = nodes[q[i]];
            const uint32_t c[2] = {nd.left, nd.right_or_first};
            for (int k = 0; k < 2; ++k)
                if (nodes[c[k]].count == 0 && m < TOP_NODES) {
                    q[m] = c[k];
                    topid[c[k]] = ++m;
                }
        }
        start = end;
        end = m;
        level_end[lv] = m;
    }
}

// Internal nodes below the top levels: they take the positions after the top levels' in the
// reference's depth-first order.
__global__ void k_wide_flags(const SrGpuNode* nodes, uint32_t n, const uint32_t* topid, uint32_t* flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = nodes[i].count == 0 && topid[i] == 0 ? 1u : 0u;
}

__device__ __forceinline__ uint32_t wide_index(const uint32_t* topid, const uint32_t* wid, uint32_t n_top, uint32_t i) {
    const uint32_t t = topid[i];
    return t ? t - 1u : n_top + wid[i];
}

// One wide node: both children's boxes in each of the `copies` sign-octant copies (near corner,
// far corner; see WideScene; copy 0 is the plain (min, max) layout), the packed child references,
// and the up links of its children (an internal child's in `up`, a leaf child's records' in
// `leafpar`: this node's index, bit 31 set for the right child).
__global__ void k_wide_fill(const SrGpuNode* nodes, uint32_t n, const uint32_t* topid, const uint32_t* wid,
                            uint32_t n_top, float4* boxes, size_t oct_stride, uint32_t copies, uint2* refs, uint32_t* up,
                            uint32_t* leafpar) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nodes[i].count != 0) return;
    const uint32_t wi = wide_index(topid, wid, n_top, i);
    const SrGpuNode& nd = nodes[i];
    uint32_t c[2] = {nd.left, nd.right_or_first}, ref[2];
    for (int k = 0; k < 2; ++k) {
        const SrGpuNode& ch = nodes[c[k]];
        for (uint32_t oct = 0; oct < copies; ++oct) {
            float nr[4], fr[4];
            for (int a = 0; a < 4; ++a) {
                const bool neg = (oct >> a) & 1u;
                nr[a] = neg ? ch.max[a] : ch.min[a];
                fr[a] = neg ? ch.min[a] : ch.max[a];
            }
            float4* b = boxes + oct * oct_stride + 4ull * wi;
            b[2 * k] = make_float4(nr[0], nr[1], nr[2], nr[3]);
            b[2 * k + 1] = make_float4(fr[0], fr[1], fr[2], fr[3]);
        }
        ref[k] = ch.count > 0 ? pack_leaf(ch.right_or_first, ch.count) : wide_index(topid, wid, n_top, c[k]);
        const uint32_t link = wi | ((uint32_t)k << 31);
        if (ch.count > 0)
            for (uint32_t p = ch.right_or_first; p < ch.right_or_first + ch.count; ++p) leafpar[p] = link;
        else
            up[ref[k]] = link;
    }
    refs[wi] = make_uint2(ref[0], ref[1]);
}

static cudaError_t lean_kernel_attrs(int max_smem);
bool lean_stack_supported(uint32_t s);

// Dynamic shared memory of the lean kernel: S + 1 stack words per thread (S of them used).
static size_t lean_stack_bytes(const SrTuning& t) {
    return t.stack_smem ? (size_t)t.block_threads * (t.stack_smem + 1) * sizeof(uint2) : 0;
}

cudaError_t fast_init(FastCtx& c, const cudaDeviceProp& prop) {
    c.num_sms = prop.multiProcessorCount;
    c.max_smem = (int)prop.sharedMemPerBlockOptin;
    return lean_kernel_attrs(c.max_smem);
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
    // Captured batch graphs hold the scene's parameters (root box, octant stride, counts) and are
    // keyed by buffer addresses that a rebuilt or re-uploaded scene can reuse: drop them all, once
    // the launches already queued on the stream have finished.
    cudaError_t e0 = cudaStreamSynchronize(st);
    if (e0 != cudaSuccess) return e0;
    fast_release(c);
    s.num_wide = 0;
    s.depth = depth;
    s.empty = n == 0;
    s.max_leaf = max_leaf;
    s.usable = depth <= FAST_MAX_DEPTH && num_prims < MAX_PACKED_PRIMS && max_leaf <= MAX_LEAF_PRIMS;
    if (n == 0 || !s.usable) return cudaSuccess;
    SrGpuNode root;
    cudaError_t e = cudaMemcpyAsync(&root, nodes, sizeof(root), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int k = 0; k < 4; ++k) { s.root_min[k] = root.min[k]; s.root_max[k] = root.max[k]; }
    if (SR_NODE_IS_NOTHING(&root)) {  // an empty tree (an arena with nothing written)
        s.empty = true;
        return cudaSuccess;
    }
    if (root.count > 0) {
        s.root_ref = pack_leaf(root.right_or_first, root.count);
        return cudaSuccess;
    }
    s.root_ref = 0;  // internal root: wide node 0 (the top levels come first)
    size_t temp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, st);
    if ((e = s.scratch.ensure(3 * (size_t)n * 4 + 64 + temp + 512)) != cudaSuccess) return e;
    uint32_t* flags = s.scratch.as<uint32_t>();
    uint32_t* wid = flags + n;
    uint32_t* topid = wid + n;
    uint32_t* level_end = topid + n;  // 16 words after topid
    uintptr_t tp = reinterpret_cast<uintptr_t>(level_end + 16);
    void* tmp = reinterpret_cast<void*>((tp + 255) & ~uintptr_t(255));
    if ((e = cudaMemsetAsync(topid, 0, (size_t)n * 4 + 64, st)) != cudaSuccess) return e;
    k_top_levels<<<1, 1, 0, st>>>(nodes, topid, level_end);
    k_wide_flags<<<(n + 255) / 256, 256, 0, st>>>(nodes, n, topid, flags);
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, temp, flags, wid, (int)n, st)) != cudaSuccess) return e;
    uint32_t last[2] = {0, 0};
    cudaMemcpyAsync(&last[0], wid + n - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last[1], flags + n - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s.top_end, level_end, sizeof(s.top_end), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    const uint32_t n_top = s.top_end[TOP_LEVELS - 1];
    s.num_wide = n_top + last[0] + last[1];
    // Box copies: 16 sign-octant copies, or one (the compact layout) when asked for, or when the
    // 15 extra copies would take more than an eighth of the device or not fit in free memory.
    const uint32_t before = s.copies;
    s.copies = 16;
    if (s.layout == SR_LAYOUT_COMPACT) {
        s.copies = 1;
    } else if (s.layout == SR_LAYOUT_AUTO) {
        size_t free_b = 0, total_b = 0;
        if ((e = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess) return e;
        const size_t one = (size_t)s.num_wide * 64;
        if (15 * one > total_b / 8 || 16 * one > free_b + s.boxes.bytes) s.copies = 1;
    }
    if (before && before != s.copies) s.boxes.release();  // a layout change does not keep the old size
    if ((e = s.boxes.ensure_grow((size_t)s.num_wide * 64 * s.copies)) != cudaSuccess) return e;
    if ((e = s.refs.ensure_grow((size_t)s.num_wide * 8)) != cudaSuccess) return e;
    if ((e = s.up.ensure_grow((size_t)s.num_wide * 4)) != cudaSuccess) return e;
    if ((e = s.leafpar.ensure_grow((size_t)num_prims * 4 + 4)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(s.up.p, 0xFF, (size_t)s.num_wide * 4, st)) != cudaSuccess) return e;  // the root: ~0
    k_wide_fill<<<(n + 255) / 256, 256, 0, st>>>(nodes, n, topid, wid, n_top, s.boxes.as<float4>(), 4ull * s.num_wide,
                                                 s.copies, s.refs.as<uint2>(), s.up.as<uint32_t>(),
                                                 s.leafpar.as<uint32_t>());
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    s.scratch.ensure(0);
    return e;
}

SrTuning fast_default_tuning(const FastCtx& c) {
    (void)c;
    SrTuning t{};
    t.block_threads = 128;
    t.blocks_per_sm = 8;  // the packet kernel's 64 registers leave room for 8 blocks of 128
    t.tile_w = 4;
    t.tile_h = 8;
    t.chunk_tiles = 1;
    t.refill_lanes = 32;
    t.leaf_coop = 0;
    t.leaf_batch = 1;
    t.home_pct = 0;
    t.packet = 1;
    return t;
}

bool fast_tuning_valid(const FastCtx& c, const SrTuning& t) {
    bool bt = t.block_threads == 64 || t.block_threads == 128 || t.block_threads == 256 || t.block_threads == 512;
    const size_t stack_bytes = lean_stack_bytes(t);
    return bt && t.blocks_per_sm >= 1 && t.blocks_per_sm <= 16 && t.tile_w >= 1 && t.tile_w * t.tile_h == 32 &&
           t.chunk_tiles >= 1 && t.chunk_tiles <= 64 && t.refill_lanes >= 1 && t.refill_lanes <= 32 &&
           t.leaf_coop <= 1 && t.leaf_batch >= 1 && t.leaf_batch <= 32 && t.home_pct <= 100 &&
           lean_stack_supported(t.stack_smem) && t.top_levels <= TOP_LEVELS &&
           (t.top_levels == 0 || t.stack_smem == 0 || t.stack_smem == 12) &&
           stack_bytes + (t.top_levels ? ((size_t)1 << t.top_levels) * 72u : 0u) <= (size_t)c.max_smem && t.packet <= 1 &&
           (t.packet == 0 || (t.stack_smem == 0 && t.top_levels == 0 && !t.leaf_coop && t.leaf_batch == 1 &&
                              t.refill_lanes == 32 && t.chunk_tiles == 1));
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

__device__ __forceinline__ void add_work(unsigned long long* c, const Work& w) {
    atomicAdd(c + 0, (unsigned long long)w.nodes);
    atomicAdd(c + 1, (unsigned long long)w.leaves);
    atomicAdd(c + 2, (unsigned long long)w.tets);
}

struct TraceBatchArgs {
    WideScene ws;
    const float4* attrs;
    const float4* mats;
    const SrGpuUniforms* U;
    const float4* cam;
    const ObsDev* obs;
    const uint32_t* tile_pre;
    uint32_t n, total_rays, tile_w, tile_h;
    uint32_t chunk_rays;    // rays a warp takes from the global counter at a time (a multiple of 32)
    uint32_t refill_lanes;  // idle lanes that make the warp fetch new rays
    uint32_t leaf_batch;    // lanes on a leaf before the warp tests leaves
    uint32_t top_n;         // lean kernel: wide nodes staged in shared memory (the top levels)
    // Lean kernel tile order: SM band b holds tiles [b * band_tiles, (b + 1) * band_tiles) and is
    // taken through sched[b]; the shared pool, tiles [num_bands * band_tiles, total), through
    // sched[num_bands].
    uint32_t num_bands, band_tiles;
    uint32_t* sched;
    float4* hits;
    uint32_t* slots;
    uint8_t* shadow;  // 0: no main-light shadow ray, 1: cast and clear, 2: cast and occluded
    uint32_t* counter;
    uint32_t* err;
    unsigned long long* work;
};

// Ray index r -> pixel: rays run tile by tile (32 consecutive rays = one tile_w x tile_h tile).
__device__ __forceinline__ bool ray_pixel(const TraceBatchArgs& a, uint32_t r, uint32_t* obs, uint32_t* px, uint32_t* py,
                                          uint32_t* p) {
    uint32_t t = r >> 5, l = r & 31u;
    uint32_t o = find_obs(a.tile_pre, a.n, t);
    const ObsDev& od = a.obs[o];
    uint32_t lt = t - __ldg(a.tile_pre + o);
    uint32_t x = (lt % od.tiles_x) * a.tile_w + l % a.tile_w;
    uint32_t y = (lt / od.tiles_x) * a.tile_h + l / a.tile_w;
    if (x >= od.width || y >= od.height) return false;
    *obs = o;
    *px = x;
    *py = y;
    *p = od.pix_base + y * od.width + x;
    return true;
}

// Shared memory of one warp for the cooperative leaf tests: the rays of the lanes at a leaf, and
// per lane the best (lambda bits << 32 | tetrahedron index in the leaf) key with its barycentrics.
constexpr uint32_t COOP_SMEM_PER_WARP = 32u * 4u * sizeof(float4) + 32u * sizeof(unsigned long long);

// Persistent traversal (see the top of the file). Each pass of the loop, with the warp converged:
//   refill     when at least `refill_lanes` lanes are idle, they take the next rays of the warp's
//              chunk (chunk_rays consecutive rays, a block of neighbouring tiles);
//   internal   every lane standing on an internal node takes one step (descend, push, or pop);
//   leaves     lanes standing on a leaf wait until `leaf_batch` lanes do (or no lane is on an
//              internal node); then the leaves are tested. With COOP the warp tests all its lanes'
//              tetrahedra together, 32 at a time, and each lane keeps the smallest lambda, ties going
//              to the first tetrahedron of the leaf, as in the sequential loop (whose test
//              `lambda >= t_max` rejects an equal lambda).
// Each ray visits exactly the nodes of the reference's traversal, in its order.
template <bool COUNT, bool COOP>
__global__ void __launch_bounds__(512) k_trace_batch(TraceBatchArgs a) {
    extern __shared__ float4 coop_smem[];
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lanes_below = (1u << lane) - 1u;
    float4* s_o = coop_smem + warp * 128u;
    float4* s_d = s_o + 32;
    float4* s_t = s_d + 32;
    float4* s_h = s_t + 32;
    unsigned long long* s_key = reinterpret_cast<unsigned long long*>(coop_smem + (blockDim.x >> 5) * 128u) + warp * 32u;

    Work wp{0, 0, 0}, wsh{0, 0, 0};
    bool has = false, occluded = false;
    uint32_t obs = 0, pix = 0, phase = 0, cur = 0, visits = 0;
    int sp = 0, slot = -1;
    float4 o = v4(0, 0, 0, 0), d = o, inv = o;
    float t_min = 0.0f, t_max = 0.0f;
    GeomHit best{0.0f, 0.0f, 0.0f, 0.0f};
    uint32_t st_ref[FAST_STACK];
    float st_t[FAST_STACK];
    uint32_t c_next = 0, c_end = 0;  // the warp's chunk (uniform across the warp)
    bool exhausted = false;          // uniform

    // Next node from the stack; primary rays skip entries entered at or beyond the closest hit.
    auto pop = [&]() -> bool {
        while (sp > 0) {
            --sp;
            if (phase != 0 || st_t[sp] < t_max) {
                cur = st_ref[sp];
                return true;
            }
        }
        return false;
    };
    // The current query is over: store its result, and start the shadow query when the main light
    // needs one.
    auto end_phase = [&]() {
        if (phase != 0) {
            a.shadow[pix] = occluded ? 2 : 1;
            has = false;
            return;
        }
        a.hits[pix] = make_float4(best.lambda, best.u, best.v, best.w);
        a.slots[pix] = slot < 0 ? 0xFFFFFFFFu : (uint32_t)slot;
        uint8_t sh_state = 0;
        has = false;
        const SrGpuUniforms& U = a.U[obs];
        if (slot >= 0 && U.mode == 0u && U.shadow_mode != 0u && U.num_flashes == 0u) {
            // compute_illumination's shadow-ray condition (renderer.rs:617-633).
            const float4* at = a.attrs + 12u * (uint32_t)slot;
            uint32_t mat = __float_as_uint(__ldg(at + 10).z);
            if (__float_as_uint(__ldg(a.mats + 3u * mat + 2u).y) == 0u) {
                float4 ev = add4(o, mul4(d, best.lambda));
                const Cam cam = cam_of(a.cam, obs);
                float4 tl;
                float dist;
                light_ray(U, cam, ev, &tl, &dist);
                if (fmaxf(rest_frame_cos(tl, __ldg(at + 8), __ldg(at + 9)), 0.0f) > 0.0f) {
                    // Bvh4D::is_occluded(hit.event, to_light, 2e-3, dist - 2e-3) (renderer.rs:636-641).
                    sh_state = 1;
                    o = ev;
                    d = tl;
                    inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
                    t_min = 2e-3f;
                    t_max = dist - 2e-3f;
                    phase = 1;
                    occluded = false;
                    visits = 0;
                    sp = 0;
                    if (slab_enter(a.ws.root_min, a.ws.root_max, o, inv, t_min, t_max) >= 0.0f) {
                        cur = a.ws.root_ref;
                        has = true;
                    }
                }
            }
        }
        if (!has) a.shadow[pix] = sh_state;
    };

    // One internal node of the lane's query: descend into the nearer child box, push the farther,
    // or pop; ends the query when the stack runs dry.
    auto node_step = [&]() {
        if (++visits > MAX_VISITS_FAST) {
            atomicOr(a.err, ERR_TRAVERSAL_LIMIT);
            sp = 0;
            end_phase();
            return;
        }
        if (COUNT) ++(phase ? wsh : wp).nodes;
        const float4* bx = a.ws.boxes + 4ull * cur;
        float4 lmin = __ldg(bx), lmax = __ldg(bx + 1), rmin = __ldg(bx + 2), rmax = __ldg(bx + 3);
        uint2 rf = __ldg(a.ws.refs + cur);
        float tl = slab_enter(lmin, lmax, o, inv, t_min, t_max);
        float tr = slab_enter(rmin, rmax, o, inv, t_min, t_max);
        bool hl = tl >= 0.0f, hr = tr >= 0.0f;
        // Primary rays cull boxes entered at or beyond the closest hit (bvh4d.rs:461); the
        // any-hit query has no such cull (bvh4d.rs:541-575) and visits left before right.
        const bool any = phase != 0;
        if (hl && hr) {
            bool left_near = any || tl <= tr;
            float tn = left_near ? tl : tr;
            if (any || tn < t_max) {
                if (sp < FAST_STACK) {
                    st_ref[sp] = left_near ? rf.y : rf.x;
                    st_t[sp] = left_near ? tr : tl;
                    ++sp;
                } else {
                    atomicOr(a.err, ERR_BAD_INDEX);
                }
                cur = left_near ? rf.x : rf.y;
                return;
            }
        } else if (hl && (any || tl < t_max)) {
            cur = rf.x;
            return;
        } else if (hr && (any || tr < t_max)) {
            cur = rf.y;
            return;
        }
        if (!pop()) end_phase();
    };

    for (;;) {
        // Refill.
        unsigned idle = __ballot_sync(FULL, !has);
        if (!exhausted && idle != 0u && (idle == FULL || (uint32_t)__popc(idle) >= a.refill_lanes)) {
            while (idle != 0u) {
                if (c_next == c_end) {
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd(a.counter, a.chunk_rays);
                    base = __shfl_sync(FULL, base, 0);
                    if (base >= a.total_rays) {
                        exhausted = true;
                        break;
                    }
                    c_next = base;
                    c_end = min(base + a.chunk_rays, a.total_rays);
                }
                uint32_t take = min(c_end - c_next, (uint32_t)__popc(idle));
                bool mine = ((idle >> lane) & 1u) && (uint32_t)__popc(idle & lanes_below) < take;
                if (mine) {
                    uint32_t r = c_next + (uint32_t)__popc(idle & lanes_below);
                    uint32_t px, py;
                    if (ray_pixel(a, r, &obs, &px, &py, &pix)) {
                        const Cam cam = cam_of(a.cam, obs);
                        float sx, sy;
                        camera_ray(a.U[obs], cam, px, py, &o, &d, &sx, &sy);
                        inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
                        t_min = 1e-3f;
                        t_max = 180.0f;
                        slot = -1;
                        phase = 0;
                        visits = 0;
                        sp = 0;
                        float re = a.ws.empty ? -1.0f : slab_enter(a.ws.root_min, a.ws.root_max, o, inv, t_min, t_max);
                        if (re >= 0.0f && re < t_max) {
                            cur = a.ws.root_ref;
                            has = true;
                        } else {  // the ray misses the scene's box (bvh4d.rs:451)
                            a.hits[pix] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                            a.slots[pix] = 0xFFFFFFFFu;
                            a.shadow[pix] = 0;
                        }
                    }
                }
                idle &= ~__ballot_sync(FULL, mine);
                c_next += take;
            }
        }

        // One internal node for every lane that stands on one.
        if (has && !(cur & REF_LEAF)) node_step();

        // Leaves: postponed until `leaf_batch` lanes stand on one, or no lane is on an internal node.
        const bool at_leaf = has && (cur & REF_LEAF);
        const unsigned lm = __ballot_sync(FULL, at_leaf);
        const unsigned nm = __ballot_sync(FULL, has && !(cur & REF_LEAF));
        if (lm == 0u) {
            if (nm == 0u && exhausted) break;
            continue;
        }
        if (nm != 0u && (uint32_t)__popc(lm) < a.leaf_batch) continue;

        if (!COOP) {
            if (at_leaf) {
                if (++visits > MAX_VISITS_FAST) {
                    atomicOr(a.err, ERR_TRAVERSAL_LIMIT);
                    sp = 0;
                } else {
                    uint32_t first = cur & REF_FIRST_MASK, cnt = (cur >> REF_COUNT_SHIFT) & 63u;
                    if (COUNT) ++(phase ? wsh : wp).leaves;
                    for (uint32_t k = first; k < first + cnt; ++k) {
                        if (COUNT) ++(phase ? wsh : wp).tets;
                        GeomHit gh;
                        if (intersect_geom(a.ws.geoms + 5u * k, o, d, t_min, t_max, &gh)) {
                            if (phase == 0) {
                                t_max = gh.lambda;
                                best = gh;
                                slot = (int)k;
                            } else {
                                occluded = true;
                                sp = 0;
                                break;
                            }
                        }
                    }
                }
                if (!pop()) end_phase();
            }
            continue;
        }
        uint32_t first = 0, cnt = 0;
        if (at_leaf) {
            if (++visits > MAX_VISITS_FAST) {
                atomicOr(a.err, ERR_TRAVERSAL_LIMIT);
                sp = 0;
            } else {
                first = cur & REF_FIRST_MASK;
                cnt = (cur >> REF_COUNT_SHIFT) & 63u;
                if (COUNT) {
                    ++(phase ? wsh : wp).leaves;
                    (phase ? wsh : wp).tets += cnt;
                }
            }
            s_o[lane] = o;
            s_d[lane] = d;
            s_t[lane] = make_float4(t_min, t_max, 0.0f, 0.0f);
            s_key[lane] = ~0ull;
        }
        uint32_t incl = cnt;
#pragma unroll
        for (uint32_t s = 1; s < 32; s <<= 1) {
            uint32_t v = __shfl_up_sync(FULL, incl, s);
            if (lane >= s) incl += v;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        const uint32_t excl = incl - cnt;
        __syncwarp();
        for (uint32_t base = 0; base < total; base += 32) {
            const uint32_t j = base + lane;
            // The owner: the first lane whose inclusive count exceeds j.
            uint32_t L = 0;
#pragma unroll
            for (uint32_t s = 16; s >= 1; s >>= 1) {
                uint32_t v = __shfl_sync(FULL, incl, L + s - 1);
                if (v <= j) L += s;
            }
            L = min(L, 31u);
            const uint32_t l_excl = __shfl_sync(FULL, excl, L);
            const uint32_t l_first = __shfl_sync(FULL, first, L);
            bool hit = false;
            unsigned long long key = 0;
            GeomHit gh;
            if (j < total) {
                const uint32_t i = j - l_excl;
                const float4 tt = s_t[L];
                if (intersect_geom(a.ws.geoms + 5u * (l_first + i), s_o[L], s_d[L], tt.x, tt.y, &gh)) {
                    key = ((unsigned long long)__float_as_uint(gh.lambda) << 32) | i;
                    atomicMin(s_key + L, key);
                    hit = true;
                }
            }
            __syncwarp();
            if (hit && s_key[L] == key) s_h[L] = make_float4(gh.u, gh.v, gh.w, 0.0f);
            __syncwarp();
        }
        if (at_leaf) {
            const unsigned long long k = s_key[lane];
            if (k != ~0ull) {
                if (phase == 0) {
                    const float4 h = s_h[lane];
                    best.lambda = __uint_as_float((uint32_t)(k >> 32));
                    best.u = h.x;
                    best.v = h.y;
                    best.w = h.z;
                    t_max = best.lambda;
                    slot = (int)(first + (uint32_t)(k & 0xFFFFFFFFull));
                } else {
                    occluded = true;
                    sp = 0;
                }
            }
            if (!pop()) end_phase();
        }
        __syncwarp();
    }
    if (COUNT) {
        add_work(a.work, wp);
        add_work(a.work + 3, wsh);
    }
}

// The default schedule (whole-tile refills, one tile per fetch, leaves tested per lane) in its lean
// form: a warp takes the next 32-ray tile when all its lanes are done, and each lane runs its
// primary query and then, when the main light needs it, its shadow query to the end, with no
// warp-wide bookkeeping per step.
__device__ __forceinline__ uint32_t sm_id() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// The next tile of a warp (called by one lane): its SM's band first, then the shared pool in
// frame order, then what is left in other SMs' bands. Returns ~0u when every tile is taken.
// `stage` and `steal` persist across calls (0: band, 1: pool, 2: stealing from band steal).
__device__ __forceinline__ uint32_t next_tile(const TraceBatchArgs& a, uint32_t home, uint32_t& stage, uint32_t& steal) {
    const uint32_t total_tiles = a.total_rays >> 5;
    if (stage == 0) {
        uint32_t v = atomicAdd(a.sched + home, 1u);
        if (v < a.band_tiles) return home * a.band_tiles + v;
        stage = 1;
    }
    const uint32_t pool_base = a.num_bands * a.band_tiles;
    if (stage == 1) {
        uint32_t v = atomicAdd(a.sched + a.num_bands, 1u);
        if (v < total_tiles - pool_base) return pool_base + v;
        stage = 2;
    }
    while (steal < a.num_bands) {
        const uint32_t b = (home + steal) % a.num_bands;
        if (*(volatile uint32_t*)(a.sched + b) < a.band_tiles) {
            uint32_t v = atomicAdd(a.sched + b, 1u);
            if (v < a.band_tiles) return b * a.band_tiles + v;
        }
        ++steal;
    }
    return ~0u;
}

// SS > 0: the first SS entries of each thread's traversal stack live in dynamic shared memory
// (SplitStack), the rest in local memory; SS == 0: all in local memory (LocalStack). OCT: the
// scene has the 16 sign-octant box copies; otherwise the compact layout (one copy). TOP: the first
// a.top_n wide nodes (the tree's top levels) are staged in shared memory after the stacks, their
// (min, max) boxes then their references. PKT: each warp walks its tile's primary rays as one
// packet (closest_packet; built with SS == 0, no staging and no counting).
template <bool COUNT, int SS, bool OCT, bool TOP, bool PKT>
__global__ void __launch_bounds__(512) k_trace_lean(const __grid_constant__ TraceBatchArgs a) {
    static_assert(!PKT || (!COUNT && SS == 0 && !TOP), "the packet form is built alone");
    const uint32_t lane = threadIdx.x & 31u;
    Work wp{0, 0, 0}, wsh{0, 0, 0};
    uint2 lm[FAST_STACK];
    extern __shared__ uint2 sm_stack[];
    using Stack = typename std::conditional<(SS > 0), SplitStack<SS>, LocalStack>::type;
    Stack st;
    if constexpr (SS > 0) st = SplitStack<SS>{sm_stack + threadIdx.x * SplitStack<SS>::ROW, lm};
    else st = LocalStack{lm};
    TopStage top{nullptr, nullptr, 0u};
    if constexpr (TOP) {
        float4* tb = reinterpret_cast<float4*>(sm_stack + (SS > 0 ? blockDim.x * (uint32_t)SplitStack<SS>::ROW : 0u));
        uint2* tr = reinterpret_cast<uint2*>(tb + 4u * a.top_n);
        for (uint32_t i = threadIdx.x; i < 4u * a.top_n; i += blockDim.x) tb[i] = __ldg(a.ws.boxes + i);  // copy 0: (min, max)
        for (uint32_t i = threadIdx.x; i < a.top_n; i += blockDim.x) tr[i] = __ldg(a.ws.refs + i);
        __syncthreads();
        top = TopStage{tb, tr, a.top_n};
    }
    const uint32_t home = a.num_bands ? sm_id() % a.num_bands : 0u;
    uint32_t stage = a.num_bands ? 0u : 1u, steal = 0;
    for (;;) {
        uint32_t tile = 0;
        if (lane == 0) tile = next_tile(a, home, stage, steal);
        tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
        if (tile == ~0u) break;
        const uint32_t base = tile << 5;
        uint32_t obs = 0, px = 0, py = 0, pix = 0;
        const bool valid = ray_pixel(a, base + lane, &obs, &px, &py, &pix);
        if (!PKT && !valid) continue;  // the packet form keeps every lane in the warp's traversal
        float4 o = v4(0.0f, 0.0f, 0.0f, 0.0f), d = v4(0.0f, 0.0f, 1.0f, 0.0f);
        if (valid) {
            float sx, sy;
            camera_ray(a.U[obs], cam_of(a.cam, obs), px, py, &o, &d, &sx, &sy);
        }
        const float4 no = neg4(o);  // the traversal and the hit event use the negated origin only
        const float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
        float t_max = 180.0f;
        GeomHit best{0.0f, 0.0f, 0.0f, 0.0f};
        int slot = -1;
        if (!a.ws.empty) {
            float en, ex;
            slab_interval(a.ws.root_min, a.ws.root_max, no, inv, 1e-3f, t_max, &en, &ex);
            const bool in = valid && ex >= en && en < t_max;  // else the ray misses the scene's box (bvh4d.rs:451)
            if constexpr (PKT) {
                if (__any_sync(0xFFFFFFFFu, in))
                    slot = closest_packet<OCT>(a.ws, in, no, d, inv, 1e-3f, t_max, best, st, a.err);
            } else if (in) {
                slot = closest_lean<COUNT, OCT, TOP>(a.ws, a.ws.root_ref, no, d, inv, 1e-3f, t_max, best, st, a.err, wp,
                                                     top);
            }
        }
        // The main light's shadow query of the pixel (compute_illumination's condition,
        // renderer.rs:617-633): per lane, or, in the packet form, the warp's queries as one packet.
        uint8_t sh = 0;
        bool shadow_in = false;
        float4 sno = v4(0.0f, 0.0f, 0.0f, 0.0f), sd = v4(0.0f, 0.0f, 1.0f, 0.0f), sinv = v4(1.0f, 1.0f, 1.0f, 1.0f);
        float s0 = 0.0f, s1 = 0.0f;
        if (valid) {
            const SrGpuUniforms& U = a.U[obs];
            a.hits[pix] = make_float4(best.lambda, best.u, best.v, best.w);
            a.slots[pix] = slot < 0 ? 0xFFFFFFFFu : (uint32_t)slot;
            if (slot >= 0 && U.mode == 0u && U.shadow_mode != 0u && U.num_flashes == 0u) {
                const float4* at = a.attrs + 12u * (uint32_t)slot;
                const uint32_t mat = __float_as_uint(__ldg(at + 10).z);
                if (__float_as_uint(__ldg(a.mats + 3u * mat + 2u).y) == 0u) {
                    const float4 ev = sub4(mul4(d, best.lambda), no);  // o + d * lambda
                    float4 tl;
                    float dist;
                    // The camera is read again here rather than kept in registers across the traversal.
                    light_ray(U, cam_of(a.cam, obs), ev, &tl, &dist);
                    if (fmaxf(rest_frame_cos(tl, __ldg(at + 8), __ldg(at + 9)), 0.0f) > 0.0f) {
                        // Bvh4D::is_occluded(hit.event, to_light, 2e-3, dist - 2e-3) (renderer.rs:636-641).
                        sh = 1;
                        sno = neg4(ev);
                        sd = tl;
                        sinv = v4(safe_inv(tl.x), safe_inv(tl.y), safe_inv(tl.z), safe_inv(tl.w));
                        s0 = 2e-3f;
                        s1 = dist - 2e-3f;
                        float en, ex;
                        slab_interval(a.ws.root_min, a.ws.root_max, sno, sinv, s0, s1, &en, &ex);
                        shadow_in = ex >= en;
                    }
                }
            }
        }
        if constexpr (PKT) {
            if (__any_sync(0xFFFFFFFFu, shadow_in) && any_packet<OCT>(a.ws, shadow_in, sno, sd, sinv, s0, s1, st, a.err))
                sh = 2;
        } else if (shadow_in && any_lean<COUNT, OCT, TOP>(a.ws, a.ws.root_ref, sno, sd, sinv, s0, s1, st, a.err, wsh, top)) {
            sh = 2;
        }
        if (valid) a.shadow[pix] = sh;
    }
    if (COUNT) {
        add_work(a.work, wp);
        add_work(a.work + 3, wsh);
    }
}

// The shared-memory stack depths the lean kernel is built for (SrTuning.stack_smem).
#define SR_LEAN_STACKS(X) X(0) X(8) X(10) X(12) X(16)

bool lean_stack_supported(uint32_t s) {
#define SR_ONE(S) if (s == (S)) return true;
    SR_LEAN_STACKS(SR_ONE)
#undef SR_ONE
    return false;
}

// The shared-memory stack and the staged top levels of the lean kernel can exceed the 48 KB
// default of one block.
template <bool COUNT, int SS, bool OCT, bool TOP>
static cudaError_t lean_attr(int max_smem) {
    return SS > 0 || TOP
               ? cudaFuncSetAttribute(k_trace_lean<COUNT, SS, OCT, TOP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      max_smem)
               : cudaSuccess;
}

template <int SS>
static cudaError_t lean_attrs_ss(int max_smem) {
    cudaError_t e = lean_attr<false, SS, true, false>(max_smem);
    if (e == cudaSuccess) e = lean_attr<true, SS, true, false>(max_smem);
    if (e == cudaSuccess) e = lean_attr<false, SS, false, false>(max_smem);
    if (e == cudaSuccess) e = lean_attr<true, SS, false, false>(max_smem);
    if constexpr (SS == 0 || SS == 12) {  // the depths built with staged top levels (octant layout)
        if (e == cudaSuccess) e = lean_attr<false, SS, true, true>(max_smem);
        if (e == cudaSuccess) e = lean_attr<true, SS, true, true>(max_smem);
    }
    return e;
}

static cudaError_t lean_kernel_attrs(int max_smem) {
    cudaError_t e = cudaSuccess;
#define SR_ONE(S) \
    if (e == cudaSuccess) e = lean_attrs_ss<(S)>(max_smem);
    SR_LEAN_STACKS(SR_ONE)
#undef SR_ONE
    return e;
}

template <int SS>
static void launch_lean_ss(bool count, bool oct, bool top, uint32_t blocks, uint32_t threads, size_t smem, cudaStream_t st,
                           const TraceBatchArgs& ta) {
    if constexpr (SS == 0 || SS == 12) {
        if (top && oct) {
            if (count) k_trace_lean<true, SS, true, true, false><<<blocks, threads, smem, st>>>(ta);
            else k_trace_lean<false, SS, true, true, false><<<blocks, threads, smem, st>>>(ta);
            return;
        }
    }
    if (oct) {
        if (count) k_trace_lean<true, SS, true, false, false><<<blocks, threads, smem, st>>>(ta);
        else k_trace_lean<false, SS, true, false, false><<<blocks, threads, smem, st>>>(ta);
    } else {
        if (count) k_trace_lean<true, SS, false, false, false><<<blocks, threads, smem, st>>>(ta);
        else k_trace_lean<false, SS, false, false, false><<<blocks, threads, smem, st>>>(ta);
    }
}

// packet: the warp-packet traversal of primary rays (counting runs always take the per-lane order,
// whose work counts are the reference traversal's).
static void launch_lean(uint32_t ss, bool count, bool oct, bool top, bool packet, uint32_t blocks, uint32_t threads,
                        size_t smem, cudaStream_t st, const TraceBatchArgs& ta) {
    if (packet && !count) {
        if (oct) k_trace_lean<false, 0, true, false, true><<<blocks, threads, smem, st>>>(ta);
        else k_trace_lean<false, 0, false, false, true><<<blocks, threads, smem, st>>>(ta);
        return;
    }
#define SR_ONE(S)                                                             \
    if (ss == (S)) {                                                          \
        launch_lean_ss<(S)>(count, oct, top, blocks, threads, smem, st, ta);  \
        return;                                                               \
    }
    SR_LEAN_STACKS(SR_ONE)
#undef SR_ONE
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
    const uint8_t* shadow;
    float4* hdr;
    uint32_t* hit_id;
    float* lambda;
    float* tau;
    uint32_t* counters;  // [0] shadow rays, [1] errors
    unsigned long long* work;
    BBConst bb;
    uint32_t stars_binned;  // observers passing stars_binned_for get their stars from k_star_tiles
};

// The shadow queries of a pixel's shading: the main light's was traced by the trace kernel (its
// state must say so); with flashes in the frame every query is traced here. The SIMPLE kernel
// (no flashes in the batch) carries no traversal code.
template <bool COUNT, bool SIMPLE>
struct FrameOccluder {
    const WideScene* s;
    uint32_t* err;
    Work* work;
    uint8_t state;
    bool trace_here;
    __device__ bool operator()(float4 o, float4 d, float t0, float t1) {
        if (!SIMPLE && trace_here) return occluded_wide<COUNT>(*s, o, d, t0, t1, err, work);
        if (state == 0) atomicOr(err, ERR_SHADOW_MISMATCH);
        return state == 2;
    }
};

// SIMPLE: every observer of the batch is flash-free and gets its stars (if any) from the binned
// pass, so the kernel has neither shadow traversal nor the per-pixel star sum.
template <bool COUNT, bool SIMPLE>
__global__ void __launch_bounds__(256, SIMPLE ? 4 : 3) k_shade_batch(const __grid_constant__ ShadeBatchArgs a) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.total_px) return;
    uint32_t o = find_obs(a.pix_pre, a.n, p);
    uint32_t l = p - __ldg(a.pix_pre + o);
    const ObsDev& od = a.obs[o];
    uint32_t px = l % od.width, py = l / od.width;
    const SrGpuUniforms& U = a.U[o];
    const Cam cam = cam_of(a.cam, o);
    float4 ro, rd;
    float sx, sy;
    camera_ray(U, cam, px, py, &ro, &rd, &sx, &sy);
    uint32_t slot = a.slots[p];
    Work work{0, 0, 0};
    uint32_t shadow_rays = 0;
    Hit h;
    h.lambda = 0.0f;
    h.tau = 0.0f;
    F3 color;
    if (slot != 0xFFFFFFFFu) {
        float4 hr = a.hits[p];
        GeomHit gh{hr.x, hr.y, hr.z, hr.w};
        interpolate(a.s.attrs + 12u * slot, ro, rd, gh, &h);
        FrameOccluder<COUNT, SIMPLE> occ{&a.ws, a.counters + 1, &work, a.shadow[p], U.num_flashes != 0u};
        color = shade_hit(a.s, U, cam, rd, h, occ, &shadow_rays);
        if (U.num_haze > 0u) color = apply_haze(color, h.event, U);
    } else {
        color = shade_sky(rd);
    }
    if (!SIMPLE && U.mode == 0u && a.s.num_stars > 0u && !(a.stars_binned && stars_binned_for(U, a.s.num_stars)))
        color = add(color, stars_brute(a.s, U, cam, ro, rd, sx, sy, slot != 0xFFFFFFFFu ? h.lambda : INFINITY, a.bb));
    a.hdr[(size_t)od.pyr_base + l] = make_float4(color.x, color.y, color.z, 0.0f);
    if (a.hit_id)
        a.hit_id[p] = slot == 0xFFFFFFFFu ? 0xFFFFFFFFu : (a.s.leaf_to_orig ? __ldg(a.s.leaf_to_orig + slot) : slot);
    if (a.lambda) a.lambda[p] = h.lambda;
    if (a.tau) a.tau[p] = h.tau;
    if (shadow_rays) atomicAdd(a.counters, shadow_rays);
    if (COUNT && work.nodes) add_work(a.work + 3, work);
}

}  // namespace srk

#include "sr_batch_bloom.cuh"
#include "sr_stars.cuh"
#include "sr_adjoint.cuh"

namespace srk {

// ---------------------------------------------------------------------------------------------
// The batch sequence.
// ---------------------------------------------------------------------------------------------
namespace {

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

struct Shape {
    uint32_t n = 0, total_tiles = 0, total_px = 0, total_pyr = 0, total_star_tiles = 0;
    std::vector<ObsDev> obs;
    std::vector<uint32_t> pre;  // (SR_BLOOM_LEVELS + 3) rows of n + 1: tiles, levels 0..6, star tiles
};

Shape make_shape(const BatchRequest& r, const SrTuning& t) {
    Shape s;
    s.n = r.n;
    s.obs.resize(r.n);
    // Rows of n + 1: trace tiles, bloom levels 0..6, 16x16 star tiles.
    const uint32_t rows = SR_BLOOM_LEVELS + 3, stride = r.n + 1;
    s.pre.assign((size_t)rows * stride, 0);
    uint32_t tiles = 0, px = 0, pyr = 0, star_tiles = 0;
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
        o.star_tile_base = star_tiles;
        s.pre[(size_t)(SR_BLOOM_LEVELS + 2) * stride + i] = star_tiles;
        star_tiles += ((o.width + STAR_TILE - 1) / STAR_TILE) * ((o.height + STAR_TILE - 1) / STAR_TILE);
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
    s.pre[(size_t)(SR_BLOOM_LEVELS + 2) * stride + r.n] = star_tiles;
    s.total_star_tiles = star_tiles;
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
    c.adj_valid = false;  // the batch buffers the gradient's outcomes live in are about to change
    Shape sh = make_shape(r, t);
    const uint32_t n = r.n, stride = n + 1;
    if ((uint64_t)sh.total_tiles * 32 >= (1ull << 32)) return cudaErrorInvalidValue;
    cudaError_t e;
    // Buffers (grown on demand; a growth invalidates every captured graph).
    size_t old_hits = c.hits.bytes, old_hdr = c.hdr.bytes, old_U = c.U.bytes, old_sh = c.shadow.bytes, old_rgb = c.rgb.bytes;
    if ((e = c.U.ensure(n * sizeof(SrGpuUniforms))) != cudaSuccess) return e;
    if ((e = c.cam64.ensure(n * sizeof(SrCameraF64))) != cudaSuccess) return e;
    if ((e = c.cam.ensure(n * 6 * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.obs.ensure(n * sizeof(ObsDev))) != cudaSuccess) return e;
    if ((e = c.lvl_pre.ensure(sh.pre.size() * 4)) != cudaSuccess) return e;
    if ((e = c.hits.ensure((size_t)sh.total_px * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.slots.ensure((size_t)sh.total_px * 4)) != cudaSuccess) return e;
    if ((e = c.shadow.ensure((size_t)sh.total_px)) != cudaSuccess) return e;  // shadow states
    if ((e = c.hdr.ensure((size_t)sh.total_pyr * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.sched.ensure(((size_t)c.num_sms + 1) * 4)) != cudaSuccess) return e;
    bool binned = false;
    if (!r.star_brute && sd.num_stars > 0)
        for (uint32_t i = 0; i < n; ++i) binned = binned || stars_binned_for(r.u[i], sd.num_stars);
    // A flash-free batch whose stars all come from the binned pass shades with the SIMPLE kernel.
    bool simple = true;
    for (uint32_t i = 0; i < n; ++i) {
        const SrGpuUniforms& ui = r.u[i];
        if (ui.num_flashes != 0u ||
            (ui.mode == 0u && sd.num_stars > 0u && !(binned && stars_binned_for(ui, sd.num_stars))))
            simple = false;
    }
    const size_t old_star = c.star_cd.bytes + c.star_rect.bytes + c.star_count.bytes + c.star_list.bytes + c.star_scan.bytes;
    // Star lists: room for every (observer, star) in 8 tiles; tiles past the room sum every star.
    const uint32_t list_cap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(8ull * n * sd.num_stars, 1u << 20), 1u << 30);
    size_t scan_bytes = 0;
    if (binned) {
        const size_t pairs = (size_t)n * sd.num_stars;
        const size_t tiles = sh.total_star_tiles;
        cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)tiles, st);
        if ((e = c.star_cd.ensure(pairs * sizeof(float4))) != cudaSuccess) return e;
        if ((e = c.star_cu.ensure(pairs * sizeof(float4))) != cudaSuccess) return e;
        if ((e = c.star_rect.ensure(pairs * sizeof(uint4))) != cudaSuccess) return e;
        if ((e = c.star_count.ensure(tiles * 4)) != cudaSuccess) return e;
        if ((e = c.star_offset.ensure(tiles * 4)) != cudaSuccess) return e;
        if ((e = c.star_fill.ensure(tiles * 4)) != cudaSuccess) return e;
        if ((e = c.star_list.ensure((size_t)list_cap * 4)) != cudaSuccess) return e;
        if ((e = c.star_scan.ensure(scan_bytes)) != cudaSuccess) return e;
    }
    if (c.star_cd.bytes + c.star_rect.bytes + c.star_count.bytes + c.star_list.bytes + c.star_scan.bytes != old_star)
        fast_release(c);
    if (!r.rgb && (e = c.rgb.ensure((size_t)sh.total_px * 4)) != cudaSuccess) return e;
    if ((e = c.hU.ensure(n * sizeof(SrGpuUniforms))) != cudaSuccess) return e;
    if ((e = c.hcam64.ensure(n * sizeof(SrCameraF64))) != cudaSuccess) return e;
    if ((e = c.hobs.ensure(n * sizeof(ObsDev))) != cudaSuccess) return e;
    if ((e = c.hlvl.ensure(sh.pre.size() * 4)) != cudaSuccess) return e;
    if (c.hits.bytes != old_hits || c.hdr.bytes != old_hdr || c.U.bytes != old_U || c.shadow.bytes != old_sh ||
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
    ws.oct_stride = 4ull * s.num_wide;
    ws.refs = s.refs.as<uint2>();
    ws.up = s.up.as<uint32_t>();
    ws.leafpar = s.leafpar.as<uint32_t>();
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
        if ((x = cudaMemsetAsync(c.sched.p, 0, c.sched.bytes, st)) != cudaSuccess) return x;
        k_camera_batch<<<(n + 63) / 64, 64, 0, st>>>(n, c.U.as<SrGpuUniforms>(), c.cam64.as<SrCameraF64>(), c.obs.as<ObsDev>(),
                                                     anchor[0], anchor[1], anchor[2], anchor[3], c.cam.as<float4>());
        if (timed) cudaEventRecord(r.ev[0], st);
        TraceBatchArgs ta;
        ta.top_n = 0;
        ta.ws = ws;
        ta.attrs = sd.attrs;
        ta.mats = sd.mats;
        ta.U = c.U.as<SrGpuUniforms>();
        ta.cam = c.cam.as<float4>();
        ta.obs = c.obs.as<ObsDev>();
        ta.tile_pre = tile_pre;
        ta.n = n;
        ta.total_rays = sh.total_tiles * 32u;
        ta.tile_w = t.tile_w;
        ta.tile_h = t.tile_h;
        ta.hits = c.hits.as<float4>();
        ta.slots = c.slots.as<uint32_t>();
        ta.shadow = c.shadow.as<uint8_t>();
        ta.chunk_rays = 32u * t.chunk_tiles;
        ta.refill_lanes = t.refill_lanes;
        ta.leaf_batch = t.leaf_batch;
        ta.counter = counters + 2;
        ta.sched = c.sched.as<uint32_t>();
        ta.num_bands = t.home_pct ? (uint32_t)c.num_sms : 0u;
        ta.band_tiles = ta.num_bands ? (uint32_t)((uint64_t)sh.total_tiles * t.home_pct / 100u / ta.num_bands) : 0u;
        if (ta.band_tiles == 0) ta.num_bands = 0;
        ta.err = counters + 1;
        ta.work = work;
        uint32_t blocks = (uint32_t)c.num_sms * t.blocks_per_sm;
        uint32_t need = (uint32_t)(((uint64_t)sh.total_tiles * 32 + t.block_threads - 1) / t.block_threads);
        if (blocks > need) blocks = need;
        const size_t smem = t.leaf_coop ? (size_t)(t.block_threads / 32) * COOP_SMEM_PER_WARP : 0;
        const bool lean = !t.leaf_coop && t.leaf_batch == 1 && t.refill_lanes == 32 && t.chunk_tiles == 1;
        if (lean) {
            // Staged top levels need the octant layout (the compact layout's kernels stage none).
            const bool oct = s.copies == 16, top = oct && t.top_levels > 0;
            ta.top_n = top ? s.top_end[t.top_levels - 1] : 0u;
            const size_t ssm = lean_stack_bytes(t) + (size_t)ta.top_n * 72u;
            launch_lean(t.stack_smem, r.count_work, oct, top, t.packet != 0, blocks, t.block_threads, ssm, st, ta);
        } else if (t.leaf_coop) {
            if (r.count_work) k_trace_batch<true, true><<<blocks, t.block_threads, smem, st>>>(ta);
            else k_trace_batch<false, true><<<blocks, t.block_threads, smem, st>>>(ta);
        } else {
            if (r.count_work) k_trace_batch<true, false><<<blocks, t.block_threads, 0, st>>>(ta);
            else k_trace_batch<false, false><<<blocks, t.block_threads, 0, st>>>(ta);
        }
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
        sa.shadow = ta.shadow;
        sa.hdr = c.hdr.as<float4>();
        sa.hit_id = r.hit_id;
        sa.lambda = r.lambda;
        sa.tau = r.tau;
        sa.counters = counters;
        sa.work = work;
        sa.bb = bb;
        sa.stars_binned = binned ? 1u : 0u;
        uint32_t gpx = (sh.total_px + 255) / 256;
        if (r.count_work) {
            if (simple) k_shade_batch<true, true><<<gpx, 256, 0, st>>>(sa);
            else k_shade_batch<true, false><<<gpx, 256, 0, st>>>(sa);
        } else {
            if (simple) k_shade_batch<false, true><<<gpx, 256, 0, st>>>(sa);
            else k_shade_batch<false, false><<<gpx, 256, 0, st>>>(sa);
        }
        if ((x = cudaGetLastError()) != cudaSuccess) return x;
        if (timed) cudaEventRecord(r.ev[2], st);
        if (binned) {
            const size_t tiles = sh.total_star_tiles;
            if ((x = cudaMemsetAsync(c.star_count.p, 0, tiles * 4, st)) != cudaSuccess) return x;
            if ((x = cudaMemsetAsync(c.star_fill.p, 0, tiles * 4, st)) != cudaSuccess) return x;
            StarBinArgs ba;
            ba.U = sa.U;
            ba.cam = sa.cam;
            ba.obs = sa.obs;
            ba.stars = sd.stars;
            ba.n = n;
            ba.num_stars = sd.num_stars;
            ba.cd = c.star_cd.as<float4>();
            ba.cu = c.star_cu.as<float4>();
            ba.rect = c.star_rect.as<uint4>();
            ba.count = c.star_count.as<uint32_t>();
            ba.offset = c.star_offset.as<uint32_t>();
            ba.fill = c.star_fill.as<uint32_t>();
            ba.list = c.star_list.as<uint32_t>();
            ba.list_cap = list_cap;
            const uint64_t pairs = (uint64_t)n * sd.num_stars;
            const uint32_t gb = (uint32_t)((pairs + 255) / 256);
            k_star_bin<<<gb, 256, 0, st>>>(ba);
            size_t sb = scan_bytes;
            if ((x = cub::DeviceScan::ExclusiveSum(c.star_scan.p, sb, ba.count, c.star_offset.as<uint32_t>(), (int)tiles, st)) !=
                cudaSuccess)
                return x;
            k_star_fill<<<gb, 256, 0, st>>>(ba);
            StarTileArgs ta2;
            ta2.s = sd;
            ta2.U = sa.U;
            ta2.cam = sa.cam;
            ta2.obs = sa.obs;
            ta2.star_pre = tile_pre + (size_t)(SR_BLOOM_LEVELS + 2) * stride;
            ta2.n = n;
            ta2.hits = sa.hits;
            ta2.slots = sa.slots;
            ta2.cd = ba.cd;
            ta2.cu = ba.cu;
            ta2.count = ba.count;
            ta2.offset = ba.offset;
            ta2.list = ba.list;
            ta2.list_cap = list_cap;
            ta2.hdr = sa.hdr;
            ta2.bb = bb;
            k_star_tiles<<<(uint32_t)tiles, 256, STAR_SORT_CAP * 4, st>>>(ta2);
            if ((x = cudaGetLastError()) != cudaSuccess) return x;
        }
        if (timed) cudaEventRecord(r.ev[3], st);
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
        const uint32_t gcomp = std::min<uint32_t>(gpx, (uint32_t)c.num_sms * 6u);
        k_bloom_composite_batch<<<gcomp, 256, 0, st>>>(sa.hdr, sa.obs, pix_pre, n, rgb, sd.tables);
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
    key = mix(key, ((uint64_t)t.chunk_tiles << 40) | ((uint64_t)t.refill_lanes << 24) | ((uint64_t)t.leaf_batch << 8) |
                       t.leaf_coop);
    key = mix(key, t.home_pct);
    key = mix(key, ((uint64_t)t.stack_smem << 32) | t.top_levels);
    key = mix(key, t.packet);
    key = mix(key, binned ? 0x5354ull : 0ull);
    key = mix(key, simple ? 0x51ull : 0ull);
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

// ---------------------------------------------------------------------------------------------
// The gradient of the image loss (sr_adjoint.cuh).
// ---------------------------------------------------------------------------------------------
cudaError_t fast_adjoint(FastCtx& c, const FastScene& s, const SrTuning& t, const SceneDev& sd, const double anchor[4],
                         const BBConst& bb, uint32_t* counters, const SrGpuUniforms& u, const SrCameraF64& cam,
                         const float* target, uint32_t level, bool frozen, uint32_t row0, uint32_t row1,
                         double out[10], cudaStream_t st) {
    const uint32_t W = u.size[0], H = u.size[1];
    cudaError_t e;
    if (frozen) {
        if (!c.adj_valid || c.adj_w != W || c.adj_h != H || c.adj_geoms != sd.geoms || c.adj_level != level ||
            c.adj_r0 != row0 || c.adj_r1 != row1)
            return cudaErrorInvalidValue;
    } else {
        // The forward frame: hits, shadow results, star lists and the HDR image the loss compares.
        BatchRequest br{};
        br.n = 1;
        br.u = &u;
        br.cam64 = &cam;
        br.use_graph = false;
        c.adj_valid = false;
        if ((e = fast_render_batch(c, s, t, sd, anchor, bb, counters, br, st)) != cudaSuccess) return e;
    }
    const uint32_t tx16 = (W + STAR_TILE - 1) / STAR_TILE, ty16 = (H + STAR_TILE - 1) / STAR_TILE;
    const uint32_t tiles = tx16 * ty16;
    const bool stars_on = sd.num_stars > 0 && stars_binned_for(u, sd.num_stars);
    // Pyramid geometry of the loss levels 0..level.
    uint32_t lw[8], lh[8];
    size_t loff[9];
    lw[0] = W;
    lh[0] = H;
    loff[0] = 0;
    for (uint32_t k = 1; k <= level; ++k) {
        lw[k] = (lw[k - 1] + 1) / 2;
        lh[k] = (lh[k - 1] + 1) / 2;
    }
    for (uint32_t k = 0; k <= level; ++k) loff[k + 1] = loff[k] + (size_t)lw[k] * lh[k];
    const size_t npx = (size_t)W * H;
    const uint32_t rblocks = (uint32_t)((npx + 255) / 256);
    const size_t list_cap = stars_on ? c.star_list.bytes / 4 : 0;
    if ((e = c.adj_cam.ensure(sizeof(DCam))) != cudaSuccess) return e;
    if ((e = c.adj_partials.ensure((size_t)std::max(tiles, rblocks) * ADJ_SLOTS * sizeof(double))) != cudaSuccess) return e;
    if ((e = c.adj_out.ensure(2 * ADJ_SLOTS * sizeof(double))) != cudaSuccess) return e;
    if ((e = c.adj_pyr.ensure(2 * loff[level + 1] * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.adj_weight.ensure(2 * npx * 3 * sizeof(double))) != cudaSuccess) return e;
    if ((e = c.adj_grid.ensure(npx)) != cudaSuccess) return e;
    if ((e = c.adj_hdr.ensure(npx * sizeof(float4))) != cudaSuccess) return e;
    if (stars_on && (e = c.adj_stars.ensure((size_t)sd.num_stars * sizeof(DF4))) != cudaSuccess) return e;
    if (stars_on && (e = c.adj_pass.ensure(list_cap * 32)) != cudaSuccess) return e;
    float4* pyr = c.adj_pyr.as<float4>();  // image levels 0..level
    float4* tpyr = pyr + loff[level + 1];  // target levels 0..level
    double* g0 = c.adj_weight.as<double>();
    double* g1 = g0 + npx * 3;
    const dim3 b2(16, 16);
    // The loss at the chosen level of `image` against the target, and (gradient mode) its weights
    // on the full image.
    auto loss_pass = [&](const void* image) -> cudaError_t {
        cudaError_t x;
        if ((x = cudaMemcpyAsync(pyr, image, npx * sizeof(float4), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return x;
        if ((x = cudaMemcpyAsync(tpyr, target, npx * sizeof(float4), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return x;
        for (uint32_t k = 1; k <= level; ++k) {
            const dim3 g2((lw[k] + 15) / 16, (lh[k] + 15) / 16);
            k_adj_down<<<g2, b2, 0, st>>>(pyr + loff[k - 1], lw[k - 1], lh[k - 1], pyr + loff[k], lw[k], lh[k]);
            k_adj_down<<<g2, b2, 0, st>>>(tpyr + loff[k - 1], lw[k - 1], lh[k - 1], tpyr + loff[k], lw[k], lh[k]);
        }
        const size_t nl = (size_t)lw[level] * lh[level];
        double* gl = (level % 2 == 0) ? g0 : g1;  // ends in g0 after `level` transposes
        const uint32_t lblocks = (uint32_t)((nl + 255) / 256);
        k_adj_residual<<<lblocks, 256, 0, st>>>(pyr + loff[level], tpyr + loff[level], (uint32_t)nl, lw[level], row0,
                                                 row1, gl, c.adj_partials.as<double>());
        k_adjoint_reduce<<<1, 256, 0, st>>>(c.adj_partials.as<double>(), lblocks, c.adj_out.as<double>() + ADJ_SLOTS);
        for (uint32_t k = level; k >= 1; --k) {
            double* src = (k % 2 == 0) ? g0 : g1;
            double* dst = (k % 2 == 0) ? g1 : g0;
            const dim3 g2((lw[k - 1] + 15) / 16, (lh[k - 1] + 15) / 16);
            k_adj_up<<<g2, b2, 0, st>>>(src, lw[k], lh[k], dst, lw[k - 1], lh[k - 1]);
        }
        return cudaGetLastError();
    };
    if (!frozen) {
        if ((e = loss_pass(c.hdr.p)) != cudaSuccess) return e;
        if (stars_on && (e = cudaMemsetAsync(c.adj_pass.p, 0, list_cap * 32, st)) != cudaSuccess) return e;
    }
    // The duals of the camera and of the stars' cone events, then the pixels.
    k_adjoint_camera<<<1, 1, 0, st>>>(cam, anchor[0], anchor[1], anchor[2], anchor[3], c.adj_cam.as<DCam>());
    if (stars_on)
        k_adjoint_stars<<<(sd.num_stars + 127) / 128, 128, 0, st>>>(sd.stars, sd.num_stars, c.adj_cam.as<DCam>(),
                                                                  c.adj_stars.as<DF4>());
    AdjointArgs a;
    a.s = sd;
    a.U = c.U.as<SrGpuUniforms>();
    a.obs = c.obs.as<ObsDev>();
    a.star_pre = nullptr;
    a.dcam = c.adj_cam.as<DCam>();
    a.hits = c.hits.as<float4>();
    a.slots = c.slots.as<uint32_t>();
    a.shadow = c.shadow.as<uint8_t>();
    a.star_dcd = stars_on ? c.adj_stars.as<DF4>() : nullptr;
    a.star_cu = stars_on ? c.star_cu.as<float4>() : nullptr;
    a.count = stars_on ? c.star_count.as<uint32_t>() : nullptr;
    a.offset = stars_on ? c.star_offset.as<uint32_t>() : nullptr;
    a.list = stars_on ? c.star_list.as<uint32_t>() : nullptr;
    a.list_cap = (uint32_t)list_cap;
    a.stars_on = stars_on ? 1u : 0u;
    a.hdr_fwd = c.hdr.as<float4>();
    a.weight = g0;
    a.partials = c.adj_partials.as<double>();
    a.bb = bb;
    a.grid = c.adj_grid.as<uint8_t>();
    a.pass = stars_on ? c.adj_pass.as<uint32_t>() : nullptr;
    a.frozen = frozen ? 1u : 0u;
    a.hdr_out = c.adj_hdr.as<float4>();
    // The band's pixel rows (level-`level` rows [row0, row1) cover rows row0 * 2^level on) and the
    // 16x16 tiles over them.
    a.y0 = std::min(H, row0 << level);
    a.y1 = std::min(H, row1 << level);
    const uint32_t ty0 = a.y0 / STAR_TILE, ty1 = (a.y1 + STAR_TILE - 1) / STAR_TILE;
    a.tile0 = ty0 * tx16;
    const uint32_t band_tiles = (ty1 - ty0) * tx16;
    if (band_tiles) k_adjoint_pixels<<<band_tiles, 256, STAR_SORT_CAP * 4, st>>>(a);
    k_adjoint_reduce<<<1, 256, 0, st>>>(a.partials, band_tiles, c.adj_out.as<double>());
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (frozen && (e = loss_pass(c.adj_hdr.p)) != cudaSuccess) return e;
    double both[2 * ADJ_SLOTS];
    if ((e = cudaMemcpyAsync(both, c.adj_out.p, sizeof(both), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    for (int k = 0; k < ADJ_SLOTS; ++k) out[k] = frozen ? 0.0 : both[k];
    out[0] = both[ADJ_SLOTS];  // the loss, from the residual pass
    if (!frozen) {
        c.adj_valid = true;
        c.adj_w = W;
        c.adj_h = H;
        c.adj_geoms = sd.geoms;
        c.adj_level = level;
        c.adj_r0 = row0;
        c.adj_r1 = row1;
    }
    return cudaSuccess;
}

}  // namespace srk
