// Traversal of the B200 node layout (shared by the batched render kernels).
//
// Layout, built on the device from the reference's GpuNode array at upload (sr_fast.cu): every
// internal node of the reference BVH2 becomes one wide node, numbered in the reference's
// depth-first order, stored as
//   boxes[i] : 64 bytes = left.min, left.max, right.min, right.max (float4 each, (t, x, y, z))
//   refs[i]  : 8 bytes  = packed child references (left, right)
// A packed reference is either a leaf, bit 31 set, bits 25..30 the primitive count (1..63) and
// bits 0..24 the first hot record; or an internal child, bit 31 clear, its wide-node index.
// Boxes are 64-byte aligned, so one traversal step reads half a cache line plus 8 bytes instead
// of the reference's three 48-byte node loads.
//
// Traversal order: near child first, the far child pushed only when both are hit, with the
// reference's culling (skip a node whose entry parameter is >= the closest hit so far). This is
// the visiting order of Bvh4D::trace (bvh4d.rs:445-520) whenever its 64-entry stack does not
// overflow (tree depth <= 60, checked at upload), so the closest hit equals the reference's,
// ties included. Any-hit queries (Bvh4D::is_occluded, bvh4d.rs:523-578) use the same layout.
#pragma once
#include "sr_device.cuh"
#include "sr_kernels.h"

namespace srk {

using namespace srd;

constexpr uint32_t REF_LEAF = 0x80000000u;
constexpr uint32_t REF_COUNT_SHIFT = 25;
constexpr uint32_t REF_FIRST_MASK = (1u << REF_COUNT_SHIFT) - 1u;
constexpr uint32_t MAX_LEAF_PRIMS = 63;
constexpr uint32_t MAX_PACKED_PRIMS = 1u << REF_COUNT_SHIFT;
constexpr uint32_t FAST_MAX_DEPTH = 60;
constexpr uint32_t MAX_VISITS_FAST = 1u << 22;
constexpr int FAST_STACK = 64;

__host__ __device__ __forceinline__ uint32_t pack_leaf(uint32_t first, uint32_t count) {
    return REF_LEAF | (count << REF_COUNT_SHIFT) | first;
}

struct WideScene {
    const float4* boxes;  // 4 float4 per wide node
    const uint2* refs;    // packed (left, right)
    const float4* geoms;  // 5 float4 per hot record
    float4 root_min, root_max;
    uint32_t root_ref;    // packed reference of the root (a leaf, or wide node 0)
    uint32_t empty;       // no geometry at all
};

// Traversal work of one thread (the SR_FLAG_COUNT_WORK variant only).
struct Work {
    uint32_t nodes, leaves, tets;
};

// Closest hit; returns the leaf slot or -1 and fills `best`.
template <bool COUNT>
__device__ __noinline__ int trace_wide(const WideScene& s, float4 o, float4 d, float t_min, float t_max, GeomHit* best,
                                       uint32_t* err, Work* work) {
    if (s.empty) return -1;
    const float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
    float re = slab_enter(s.root_min, s.root_max, o, inv, t_min, t_max);
    if (re < 0.0f || re >= t_max) return -1;
    uint32_t cur = s.root_ref;
    int slot = -1;
    uint32_t st_ref[FAST_STACK];
    float st_t[FAST_STACK];
    int sp = 0;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MAX_VISITS_FAST) { atomicOr(err, ERR_TRAVERSAL_LIMIT); break; }
        bool descend = false;
        if (!(cur & REF_LEAF)) {
            if (COUNT) ++work->nodes;
            const float4* b = s.boxes + 4ull * cur;
            float4 lmin = __ldg(b), lmax = __ldg(b + 1), rmin = __ldg(b + 2), rmax = __ldg(b + 3);
            uint2 r = __ldg(s.refs + cur);
            float tl = slab_enter(lmin, lmax, o, inv, t_min, t_max);
            float tr = slab_enter(rmin, rmax, o, inv, t_min, t_max);
            bool hl = tl >= 0.0f, hr = tr >= 0.0f;
            if (hl && hr) {
                bool left_near = tl <= tr;
                float tn = left_near ? tl : tr;
                if (tn < t_max) {
                    if (sp < FAST_STACK) {
                        st_ref[sp] = left_near ? r.y : r.x;
                        st_t[sp] = left_near ? tr : tl;
                        ++sp;
                    } else {
                        atomicOr(err, ERR_BAD_INDEX);
                    }
                    cur = left_near ? r.x : r.y;
                    descend = true;
                }
            } else if (hl) {
                if (tl < t_max) { cur = r.x; descend = true; }
            } else if (hr) {
                if (tr < t_max) { cur = r.y; descend = true; }
            }
        } else {
            uint32_t first = cur & REF_FIRST_MASK, cnt = (cur >> REF_COUNT_SHIFT) & 63u;
            if (COUNT) { ++work->leaves; work->tets += cnt; }
            for (uint32_t k = first; k < first + cnt; ++k) {
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
            if (st_t[sp] < t_max) { cur = st_ref[sp]; found = true; break; }
        }
        if (!found) break;
    }
    return slot;
}

// Any hit in (t_min, t_max).
template <bool COUNT>
__device__ __noinline__ bool occluded_wide(const WideScene& s, float4 o, float4 d, float t_min, float t_max, uint32_t* err,
                                           Work* work) {
    if (s.empty) return false;
    const float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
    if (slab_enter(s.root_min, s.root_max, o, inv, t_min, t_max) < 0.0f) return false;
    uint32_t cur = s.root_ref;
    uint32_t st_ref[FAST_STACK];
    int sp = 0;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MAX_VISITS_FAST) { atomicOr(err, ERR_TRAVERSAL_LIMIT); return false; }
        bool descend = false;
        if (!(cur & REF_LEAF)) {
            if (COUNT) ++work->nodes;
            const float4* b = s.boxes + 4ull * cur;
            float4 lmin = __ldg(b), lmax = __ldg(b + 1), rmin = __ldg(b + 2), rmax = __ldg(b + 3);
            uint2 r = __ldg(s.refs + cur);
            bool hl = slab_enter(lmin, lmax, o, inv, t_min, t_max) >= 0.0f;
            bool hr = slab_enter(rmin, rmax, o, inv, t_min, t_max) >= 0.0f;
            if (hl && hr) {
                if (sp < FAST_STACK) st_ref[sp++] = r.y; else atomicOr(err, ERR_BAD_INDEX);
                cur = r.x;
                descend = true;
            } else if (hl) {
                cur = r.x;
                descend = true;
            } else if (hr) {
                cur = r.y;
                descend = true;
            }
        } else {
            uint32_t first = cur & REF_FIRST_MASK, cnt = (cur >> REF_COUNT_SHIFT) & 63u;
            if (COUNT) ++work->leaves;
            for (uint32_t k = first; k < first + cnt; ++k) {
                if (COUNT) ++work->tets;
                GeomHit gh;
                if (intersect_geom(s.geoms + 5u * k, o, d, t_min, t_max, &gh)) return true;
            }
        }
        if (descend) continue;
        if (sp == 0) return false;
        cur = st_ref[--sp];
    }
}

}  // namespace srk
