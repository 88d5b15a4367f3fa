// The fast path.
//
// Node layout: each internal node of the reference BVH2 becomes one 80-byte wide node holding
// both children's boxes (five 16-byte loads), built on the device at upload. A traversal step
// costs one node fetch instead of the reference's three (node, left box, right box).
//
// Traversal: near child first, far child pushed only when both children are hit, with the
// reference's culling (a node is skipped when its entry parameter is >= the closest hit so far).
// This visits nodes and tests tetrahedra in exactly the order of Bvh4D::trace (bvh4d.rs:445-520)
// whenever the reference's 64-entry stack does not overflow (tree depth <= 60, checked at upload;
// deeper trees render on the plain path), so the closest hit is the reference's, ties included.
//
// Kernels: a persistent trace kernel (one warp takes a 32-pixel tile at a time from a global
// counter) writes the primary hit records; the shade kernel interpolates, shades, casts shadow
// rays over the same layout and adds the star term. Splitting them keeps the traversal kernel's
// register count, and with it its occupancy, independent of the branch-heavy clock textures.
#include <cub/cub.cuh>

#include "sr_fast.h"
#include "sr_shade.cuh"

namespace srk {

using namespace srd;

constexpr uint32_t FAST_MAX_DEPTH = 60;
constexpr uint32_t MAX_VISITS_FAST = 1u << 22;
constexpr int FAST_STACK = 64;

__global__ void k_wide_flags(const SrGpuNode* nodes, uint32_t n, uint32_t* flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = nodes[i].count == 0 ? 1u : 0u;
}

__global__ void k_wide_fill(const SrGpuNode* nodes, uint32_t n, const uint32_t* wid, uint4* wide) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nodes[i].count != 0) return;
    const SrGpuNode& nd = nodes[i];
    uint32_t c[2] = {nd.left, nd.right_or_first};
    uint4* w = wide + 5ull * wid[i];
    uint32_t ref[2], cnt[2];
    for (int k = 0; k < 2; ++k) {
        const SrGpuNode& ch = nodes[c[k]];
        w[2 * k] = make_uint4(__float_as_uint(ch.min[0]), __float_as_uint(ch.min[1]), __float_as_uint(ch.min[2]), __float_as_uint(ch.min[3]));
        w[2 * k + 1] = make_uint4(__float_as_uint(ch.max[0]), __float_as_uint(ch.max[1]), __float_as_uint(ch.max[2]), __float_as_uint(ch.max[3]));
        ref[k] = ch.count > 0 ? ch.right_or_first : wid[c[k]];
        cnt[k] = ch.count;
    }
    w[4] = make_uint4(ref[0], ref[1], cnt[0], cnt[1]);
}

cudaError_t fast_init(FastCtx& c, const cudaDeviceProp& prop) {
    c.num_sms = prop.multiProcessorCount;
    c.max_smem = (int)prop.sharedMemPerBlockOptin;
    return cudaSuccess;
}

void fast_release(FastCtx& c) {
    c.hits.ensure(0);
    c.slots.ensure(0);
}

cudaError_t fast_build(FastCtx& c, FastScene& s, const SrGpuNode* nodes, uint32_t n, uint32_t depth, cudaStream_t st) {
    (void)c;
    s.num_wide = 0;
    s.depth = depth;
    s.root_is_leaf = false;
    if (n == 0) return cudaSuccess;
    SrGpuNode root;
    cudaError_t e = cudaMemcpyAsync(&root, nodes, sizeof(root), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int k = 0; k < 4; ++k) { s.root_min[k] = root.min[k]; s.root_max[k] = root.max[k]; }
    if (root.count > 0) {
        s.root_is_leaf = true;
        s.root_first = root.right_or_first;
        s.root_count = root.count;
        return cudaSuccess;
    }
    size_t temp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, st);
    size_t need = 2 * (size_t)n * 4 + temp + 256;
    if ((e = s.scratch.ensure(need)) != cudaSuccess) return e;
    uint32_t* flags = s.scratch.as<uint32_t>();
    uint32_t* wid = flags + n;
    void* tmp = reinterpret_cast<char*>(wid + n) + (256 - ((uintptr_t)(wid + n) & 255));
    k_wide_flags<<<(n + 255) / 256, 256, 0, st>>>(nodes, n, flags);
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, temp, flags, wid, (int)n, st)) != cudaSuccess) return e;
    uint32_t last_wid = 0, last_flag = 0;
    cudaMemcpyAsync(&last_wid, wid + n - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_flag, flags + n - 1, 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    s.num_wide = last_wid + last_flag;
    if ((e = s.wide.ensure((size_t)s.num_wide * 80)) != cudaSuccess) return e;
    k_wide_fill<<<(n + 255) / 256, 256, 0, st>>>(nodes, n, wid, s.wide.as<uint4>());
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    s.scratch.ensure(0);
    return cudaStreamSynchronize(st);
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
    return bt && t.blocks_per_sm >= 1 && t.blocks_per_sm <= 16 && t.tile_w * t.tile_h == 32 && t.tile_w >= 1 &&
           t.stack_depth == (uint32_t)FAST_STACK && t.smem_levels == 0;
}

struct WideScene {
    const uint4* wide;
    const float4* geoms;
    uint32_t num_wide;
    uint32_t root_is_leaf, root_first, root_count;
    float4 root_min, root_max;
};

__device__ __forceinline__ void load_wide(const uint4* w, uint32_t i, float4* lmin, float4* lmax, float4* rmin,
                                          float4* rmax, uint4* meta) {
    const uint4* p = w + 5ull * i;
    uint4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    *meta = __ldg(p + 4);
    *lmin = make_float4(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z), __uint_as_float(a.w));
    *lmax = make_float4(__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z), __uint_as_float(b.w));
    *rmin = make_float4(__uint_as_float(c.x), __uint_as_float(c.y), __uint_as_float(c.z), __uint_as_float(c.w));
    *rmax = make_float4(__uint_as_float(d.x), __uint_as_float(d.y), __uint_as_float(d.z), __uint_as_float(d.w));
}

// Traversal work of one thread (the SR_FLAG_COUNT_WORK variant only).
struct Work {
    uint32_t nodes, leaves, tets;
};

// Closest hit over the wide layout; returns the leaf slot or -1.
template <bool COUNT>
__device__ __noinline__ int trace_fast(const WideScene& s, float4 o, float4 d, float t_min, float t_max, GeomHit* best,
                                       uint32_t* err, Work* work) {
    float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
    int slot = -1;
    uint32_t cur, cur_cnt;
    if (s.root_is_leaf) {
        float re = slab_enter(s.root_min, s.root_max, o, inv, t_min, t_max);
        if (re < 0.0f || re >= t_max) return -1;
        cur = s.root_first;
        cur_cnt = s.root_count;
    } else {
        if (s.num_wide == 0u) return -1;
        float re = slab_enter(s.root_min, s.root_max, o, inv, t_min, t_max);
        if (re < 0.0f || re >= t_max) return -1;
        cur = 0;
        cur_cnt = 0;
    }
    uint32_t st_ref[FAST_STACK], st_cnt[FAST_STACK];
    float st_t[FAST_STACK];
    int sp = 0;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MAX_VISITS_FAST) { atomicOr(err, ERR_TRAVERSAL_LIMIT); break; }
        bool descend = false;
        if (cur_cnt == 0u) {
            if (COUNT) ++work->nodes;
            float4 lmin, lmax, rmin, rmax;
            uint4 m;
            load_wide(s.wide, cur, &lmin, &lmax, &rmin, &rmax, &m);
            float tl = slab_enter(lmin, lmax, o, inv, t_min, t_max);
            float tr = slab_enter(rmin, rmax, o, inv, t_min, t_max);
            bool hl = tl >= 0.0f, hr = tr >= 0.0f;
            if (hl && hr) {
                bool left_near = tl <= tr;
                float tn = left_near ? tl : tr, tf = left_near ? tr : tl;
                if (tn < t_max) {
                    if (sp < FAST_STACK) {
                        st_ref[sp] = left_near ? m.y : m.x;
                        st_cnt[sp] = left_near ? m.w : m.z;
                        st_t[sp] = tf;
                        ++sp;
                    } else {
                        atomicOr(err, ERR_BAD_INDEX);
                    }
                    cur = left_near ? m.x : m.y;
                    cur_cnt = left_near ? m.z : m.w;
                    descend = true;
                }
            } else if (hl) {
                if (tl < t_max) { cur = m.x; cur_cnt = m.z; descend = true; }
            } else if (hr) {
                if (tr < t_max) { cur = m.y; cur_cnt = m.w; descend = true; }
            }
        } else {
            if (COUNT) { ++work->leaves; work->tets += cur_cnt; }
            for (uint32_t k = cur; k < cur + cur_cnt; ++k) {
                GeomHit gh;
                if (intersect_geom(s.geoms + 5u * k, o, d, t_min, t_max, &gh)) {
                    t_max = gh.lambda;
                    *best = gh;
                    slot = (int)k;
                }
            }
        }
        if (descend) continue;
        bool found = false;
        while (sp > 0) {
            --sp;
            if (st_t[sp] < t_max) { cur = st_ref[sp]; cur_cnt = st_cnt[sp]; found = true; break; }
        }
        if (!found) break;
    }
    return slot;
}

// Any hit in (t_min, t_max) over the wide layout (Bvh4D::is_occluded, bvh4d.rs:523-578).
template <bool COUNT>
__device__ __noinline__ bool occluded_fast(const WideScene& s, float4 o, float4 d, float t_min, float t_max, uint32_t* err,
                                           Work* work) {
    float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
    if (slab_enter(s.root_min, s.root_max, o, inv, t_min, t_max) < 0.0f) return false;
    uint32_t cur = s.root_is_leaf ? s.root_first : 0u, cur_cnt = s.root_is_leaf ? s.root_count : 0u;
    if (!s.root_is_leaf && s.num_wide == 0u) return false;
    uint32_t st_ref[FAST_STACK], st_cnt[FAST_STACK];
    int sp = 0;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MAX_VISITS_FAST) { atomicOr(err, ERR_TRAVERSAL_LIMIT); return false; }
        bool descend = false;
        if (cur_cnt == 0u) {
            if (COUNT) ++work->nodes;
            float4 lmin, lmax, rmin, rmax;
            uint4 m;
            load_wide(s.wide, cur, &lmin, &lmax, &rmin, &rmax, &m);
            bool hl = slab_enter(lmin, lmax, o, inv, t_min, t_max) >= 0.0f;
            bool hr = slab_enter(rmin, rmax, o, inv, t_min, t_max) >= 0.0f;
            if (hl && hr) {
                if (sp < FAST_STACK) { st_ref[sp] = m.y; st_cnt[sp] = m.w; ++sp; } else atomicOr(err, ERR_BAD_INDEX);
                cur = m.x; cur_cnt = m.z; descend = true;
            } else if (hl) {
                cur = m.x; cur_cnt = m.z; descend = true;
            } else if (hr) {
                cur = m.y; cur_cnt = m.w; descend = true;
            }
        } else {
            if (COUNT) ++work->leaves;
            for (uint32_t k = cur; k < cur + cur_cnt; ++k) {
                if (COUNT) ++work->tets;
                GeomHit gh;
                if (intersect_geom(s.geoms + 5u * k, o, d, t_min, t_max, &gh)) return true;
            }
        }
        if (descend) continue;
        if (sp == 0) return false;
        --sp;
        cur = st_ref[sp];
        cur_cnt = st_cnt[sp];
    }
}

template <bool COUNT>
struct FastOccluder {
    const WideScene* s;
    uint32_t* err;
    Work* work;
    __device__ bool operator()(float4 o, float4 d, float t0, float t1) {
        return occluded_fast<COUNT>(*s, o, d, t0, t1, err, work);
    }
};

// Adds a warp's work to the 64-bit counters (counting variant only).
__device__ __forceinline__ void add_work(unsigned long long* c, const Work& w) {
    atomicAdd(c + 0, (unsigned long long)w.nodes);
    atomicAdd(c + 1, (unsigned long long)w.leaves);
    atomicAdd(c + 2, (unsigned long long)w.tets);
}

struct TraceArgs {
    WideScene ws;
    uint32_t width, height, tile_w, tile_h, tiles_x, n_tiles;
    float4* hit;
    uint32_t* slot;
    uint32_t* counter;
    uint32_t* err;
    unsigned long long* work;  // 6 counters (primary nodes, leaves, tets; shadow nodes, leaves, tets)
};

// Persistent primary-ray kernel: each warp takes a tile_w x tile_h tile of pixels at a time.
template <bool COUNT>
__global__ void __launch_bounds__(512) k_trace_fast(TraceArgs a, SrGpuUniforms U, const float4* cam_dev) {
    const uint32_t lane = threadIdx.x & 31u;
    const Cam cam = load_cam(U, cam_dev);
    Work work{0, 0, 0};
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(a.counter, 1u);
        t = __shfl_sync(0xFFFFFFFFu, t, 0);
        if (t >= a.n_tiles) break;
        uint32_t px = (t % a.tiles_x) * a.tile_w + lane % a.tile_w;
        uint32_t py = (t / a.tiles_x) * a.tile_h + lane / a.tile_w;
        if (px >= a.width || py >= a.height) continue;
        float4 o, d;
        float sx, sy;
        camera_ray(U, cam, px, py, &o, &d, &sx, &sy);
        GeomHit gh;
        int slot = trace_fast<COUNT>(a.ws, o, d, 1e-3f, 180.0f, &gh, a.err, &work);
        size_t idx = (size_t)py * a.width + px;
        a.hit[idx] = make_float4(gh.lambda, gh.u, gh.v, gh.w);
        a.slot[idx] = slot < 0 ? 0xFFFFFFFFu : (uint32_t)slot;
    }
    if (COUNT) add_work(a.work, work);
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_shade_fast(SceneDev s, WideScene ws, SrGpuUniforms U, const float4* cam_dev,
                                                     FrameDev f, const float4* hits, const uint32_t* slots, BBConst bb,
                                                     unsigned long long* work_out) {
    uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= U.size[0] || py >= U.size[1]) return;
    const Cam cam = load_cam(U, cam_dev);
    size_t idx = (size_t)py * U.size[0] + px;
    float4 o, d;
    float sx, sy;
    camera_ray(U, cam, px, py, &o, &d, &sx, &sy);
    uint32_t slot = slots[idx];
    uint32_t shadow_rays = 0;
    F3 color;
    Hit h;
    h.lambda = 0.0f;
    h.tau = 0.0f;
    if (slot != 0xFFFFFFFFu) {
        float4 hr = hits[idx];
        GeomHit gh{hr.x, hr.y, hr.z, hr.w};
        interpolate(s.attrs + 12u * slot, o, d, gh, &h);
        Work work{0, 0, 0};
        FastOccluder<COUNT> occ{&ws, f.counters + 1, &work};
        color = shade_hit(s, U, cam, d, h, occ, &shadow_rays);
        if (U.num_haze > 0u) color = apply_haze(color, h.event, U);
        if (COUNT && work.nodes) add_work(work_out + 3, work);
    } else {
        color = shade_sky(d);
    }
    if (U.mode == 0u && s.num_stars > 0u)
        color = add(color, stars_brute(s, U, cam, o, d, sx, sy, slot != 0xFFFFFFFFu ? h.lambda : INFINITY, bb));
    f.hdr[idx] = make_float4(color.x, color.y, color.z, 0.0f);
    if (f.hit_id) f.hit_id[idx] = slot == 0xFFFFFFFFu ? 0xFFFFFFFFu : (s.leaf_to_orig ? __ldg(s.leaf_to_orig + slot) : slot);
    if (f.lambda) f.lambda[idx] = h.lambda;
    if (f.tau) f.tau[idx] = h.tau;
    if (shadow_rays) atomicAdd(f.counters, shadow_rays);
}

cudaError_t fast_render(FastCtx& c, const FastScene& s, const SrTuning& t, const SceneDev& sd, const SrGpuUniforms& u,
                        const float4* cam_dev, const FrameDev& f, const BBConst& bb, cudaStream_t st, cudaEvent_t* ev,
                        bool count_work) {
    if (s.depth > FAST_MAX_DEPTH) {
        // The reference's 64-entry stack may overflow and drop children on such trees; the plain
        // path reproduces that exactly.
        cudaError_t e = launch_render_plain(sd, u, cam_dev, f, bb, st);
        if (ev) { cudaEventRecord(ev[0], st); cudaEventRecord(ev[1], st); }
        return e;
    }
    size_t npx = (size_t)u.size[0] * u.size[1];
    cudaError_t e;
    if ((e = c.hits.ensure(npx * sizeof(float4))) != cudaSuccess) return e;
    if ((e = c.slots.ensure(npx * 4)) != cudaSuccess) return e;
    WideScene ws;
    ws.wide = s.wide.as<uint4>();
    ws.geoms = sd.geoms;
    ws.num_wide = s.num_wide;
    ws.root_is_leaf = s.root_is_leaf ? 1u : 0u;
    ws.root_first = s.root_first;
    ws.root_count = s.root_count;
    ws.root_min = make_float4(s.root_min[0], s.root_min[1], s.root_min[2], s.root_min[3]);
    ws.root_max = make_float4(s.root_max[0], s.root_max[1], s.root_max[2], s.root_max[3]);
    if (sd.num_nodes == 0) { ws.num_wide = 0; ws.root_is_leaf = 0; ws.root_min = make_float4(1, 1, 1, 1); ws.root_max = make_float4(-1, -1, -1, -1); }
    TraceArgs a;
    a.ws = ws;
    a.width = u.size[0];
    a.height = u.size[1];
    a.tile_w = t.tile_w;
    a.tile_h = t.tile_h;
    a.tiles_x = (u.size[0] + t.tile_w - 1) / t.tile_w;
    a.n_tiles = a.tiles_x * ((u.size[1] + t.tile_h - 1) / t.tile_h);
    a.hit = c.hits.as<float4>();
    a.slot = c.slots.as<uint32_t>();
    a.counter = f.counters + 2;
    a.err = f.counters + 1;
    a.work = reinterpret_cast<unsigned long long*>(f.counters + 4);
    uint32_t blocks = (uint32_t)c.num_sms * t.blocks_per_sm;
    uint32_t max_blocks = (a.n_tiles * 32 + t.block_threads - 1) / t.block_threads;
    if (blocks > max_blocks) blocks = max_blocks;
    if (count_work) k_trace_fast<true><<<blocks, t.block_threads, 0, st>>>(a, u, cam_dev);
    else k_trace_fast<false><<<blocks, t.block_threads, 0, st>>>(a, u, cam_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[0], st);
    dim3 b(16, 16), g((u.size[0] + 15) / 16, (u.size[1] + 15) / 16);
    if (count_work)
        k_shade_fast<true><<<g, b, 0, st>>>(sd, ws, u, cam_dev, f, c.hits.as<float4>(), c.slots.as<uint32_t>(), bb, a.work);
    else
        k_shade_fast<false><<<g, b, 0, st>>>(sd, ws, u, cam_dev, f, c.hits.as<float4>(), c.slots.as<uint32_t>(), bb, a.work);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[1], st);
    return cudaSuccess;
}

}  // namespace srk
