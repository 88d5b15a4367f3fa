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
// of the reference's three 48-byte node loads. Numbering: the internal nodes of the top
// TOP_LEVELS levels first, breadth first, then the others in the reference's depth-first order.
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
constexpr uint32_t REF_COUNT_MASK = 63u << REF_COUNT_SHIFT;
// Adding this to a leaf reference moves it past its first primitive: first + 1, count - 1 (first
// + count never reaches 2^25, so the fields do not carry into each other).
constexpr uint32_t REF_NEXT_PRIM = 1u - (1u << REF_COUNT_SHIFT);
constexpr uint32_t MAX_LEAF_PRIMS = 63;
constexpr uint32_t MAX_PACKED_PRIMS = 1u << REF_COUNT_SHIFT;
constexpr uint32_t FAST_MAX_DEPTH = 60;
constexpr uint32_t MAX_VISITS_FAST = 1u << 22;
constexpr int FAST_STACK = 64;
// The wide nodes of the tree's top TOP_LEVELS levels come first, level by level (breadth first),
// so the top K levels are the prefix [0, top_end[K - 1]) for every K <= TOP_LEVELS; the lean
// kernel can stage such a prefix in shared memory (SrTuning::top_levels).
constexpr uint32_t TOP_LEVELS = 8;
constexpr uint32_t TOP_NODES = (1u << TOP_LEVELS) - 1u;

__host__ __device__ __forceinline__ uint32_t pack_leaf(uint32_t first, uint32_t count) {
    return REF_LEAF | (count << REF_COUNT_SHIFT) | first;
}

struct WideScene {
    // 16 copies of the child boxes, one per sign octant of the inverse direction (bit i set: the
    // ray's inv component i is negative). In copy `oct` each child holds its near corner then its
    // far corner: component i is min[i] for a positive inv[i], max[i] for a negative one. Copy 0
    // is therefore the plain (min, max) layout. 4 float4 per wide node in each copy.
    const float4* boxes;
    size_t oct_stride;    // float4 count of one copy (4 per wide node)
    const uint2* refs;    // packed (left, right)
    const float4* geoms;  // 5 float4 per hot record
    // Up links, for ordering two hits of equal lambda the way the reference's traversal meets them
    // (packet traversal only): up[w] = parent wide node of wide node w | side << 31 (side 1: the
    // right child), ~0u for the root; leafpar[k] = the same for the leaf holding hot record k.
    const uint32_t* up;
    const uint32_t* leafpar;
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

// ---------------------------------------------------------------------------------------------
// The lean forms used by the persistent batch kernel. Same visiting order and the same values as
// trace_wide / occluded_wide; fewer instructions per step:
//   - the five-way max / min of the slab test use the three-input max.f32 / min.f32 of sm_100
//     (max and min are exact, the inputs are never NaN: inv is never 0 and boxes are finite);
//   - a child is taken when its slab interval is non-empty and, for closest-hit queries, entered
//     before the closest hit. The far child of a pair is therefore not pushed when it is entered
//     at or beyond the closest hit; the reference pushes it and discards it when popped, so the
//     nodes visited are the same;
//   - a stack entry is one 8-byte word (reference, entry parameter bits);
//   - the slab and tetrahedron arithmetic runs in paired fp32 instructions (below).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Paired fp32 arithmetic of sm_100 (add / mul .rn.f32x2): each half is the IEEE round-to-nearest
// result of the scalar operation, so these give the scalar code's values bit for bit, as long as
// no paired product feeds a paired sum (ptxas fuses that pair into one fma even with --fmad=false
// and explicit rounding; the code below never forms it). `a - b` is computed as `a + (-b)`, which
// IEEE 754 defines to be the same operation.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "add.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mul.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
// edot (minkowski.rs:198-200): ((a.t b.t + a.x b.x) + a.y b.y) + a.z b.z.
__device__ __forceinline__ float edot_p(float4 a, float4 b) {
    const float2 p = mul2(f2(a.x, a.y), f2(b.x, b.y)), q = mul2(f2(a.z, a.w), f2(b.z, b.w));
    return ((p.x + p.y) + q.x) + q.y;
}

// Entry and exit parameters of the slab test (Aabb4D::intersect_ray, mesh4d.rs:114-146) for a ray
// with origin -no: the box is hit when exit >= entry; entry >= t_min > 0.
__device__ __forceinline__ void slab_interval(float4 bmin, float4 bmax, float4 no, float4 inv, float t_min, float t_max,
                                              float* en, float* ex) {
    const float2 i01 = f2(inv.x, inv.y), i23 = f2(inv.z, inv.w);
    const float2 a01 = mul2(add2(f2(bmin.x, bmin.y), f2(no.x, no.y)), i01);
    const float2 a23 = mul2(add2(f2(bmin.z, bmin.w), f2(no.z, no.w)), i23);
    const float2 b01 = mul2(add2(f2(bmax.x, bmax.y), f2(no.x, no.y)), i01);
    const float2 b23 = mul2(add2(f2(bmax.z, bmax.w), f2(no.z, no.w)), i23);
    *en = max3f(max3f(t_min, fminf(a01.x, b01.x), fminf(a01.y, b01.y)), fminf(a23.x, b23.x), fminf(a23.y, b23.y));
    *ex = min3f(min3f(t_max, fmaxf(a01.x, b01.x), fmaxf(a01.y, b01.y)), fmaxf(a23.x, b23.x), fmaxf(a23.y, b23.y));
}

// SimplexGeom4D::intersect_fast (mesh4d.rs:175-211) in paired arithmetic, for a ray with origin
// o = -no: the values of intersect_geom bit for bit.
__device__ __forceinline__ bool intersect_lean(const float4* g, float4 no, float4 d, float t_min, float t_max,
                                               GeomHit* h) {
    const float4 n = __ldg(g + 1);
    const float denom = edot_p(n, d);
    if (fabsf(denom) < 1e-9f) return false;
    const float4 v0 = __ldg(g);
    const float2 w01 = add2(f2(v0.x, v0.y), f2(no.x, no.y)), w23 = add2(f2(v0.z, v0.w), f2(no.z, no.w));
    const float lambda = edot_p(n, make_float4(w01.x, w01.y, w23.x, w23.y)) / denom;
    if (lambda <= t_min || lambda >= t_max) return false;
    // The event o + d * lambda in scalar arithmetic: ptxas fuses a paired product followed by a
    // paired sum into one fused multiply-add (one rounding), whatever the rounding modifiers say.
    const float4 ev = sub4(mul4(d, lambda), no);  // o + d * lambda: negation is exact, a - b is a + (-b)
    const float2 q01 = add2(f2(ev.x, ev.y), f2(-v0.x, -v0.y)), q23 = add2(f2(ev.z, ev.w), f2(-v0.z, -v0.w));
    const float4 q = make_float4(q01.x, q01.y, q23.x, q23.y);
    const float eps = -1e-5f;
    const float u = edot_p(__ldg(g + 2), q);
    if (u < eps || u > 1.0f - eps) return false;
    const float v = edot_p(__ldg(g + 3), q);
    if (v < eps || u + v > 1.0f - eps) return false;
    const float w = edot_p(__ldg(g + 4), q);
    if (w < eps || u + v + w > 1.0f - eps) return false;
    h->lambda = lambda;
    h->u = u;
    h->v = v;
    h->w = w;
    return true;
}

// The same interval from a box stored near corner first for the ray's sign octant: the near
// plane's parameter of each axis is then the smaller one (the products keep the order of the
// sums, rounding being monotonic, since the sign of inv is the octant's), so the per-axis min and
// max of slab_interval are not needed and the values are the same bit for bit.
__device__ __forceinline__ void slab_octant(float4 bnear, float4 bfar, float4 no, float4 inv, float t_min, float t_max,
                                            float* en, float* ex) {
    const float2 i01 = f2(inv.x, inv.y), i23 = f2(inv.z, inv.w);
    const float2 a01 = mul2(add2(f2(bnear.x, bnear.y), f2(no.x, no.y)), i01);
    const float2 a23 = mul2(add2(f2(bnear.z, bnear.w), f2(no.z, no.w)), i23);
    const float2 b01 = mul2(add2(f2(bfar.x, bfar.y), f2(no.x, no.y)), i01);
    const float2 b23 = mul2(add2(f2(bfar.z, bfar.w), f2(no.z, no.w)), i23);
    *en = max3f(max3f(t_min, a01.x, a01.y), a23.x, a23.y);
    *ex = min3f(min3f(t_max, b01.x, b01.y), b23.x, b23.y);
}

// The box copy of a ray's sign octant (safe_inv never returns 0, so inv < 0 is the sign).
__device__ __forceinline__ const float4* octant_boxes(const WideScene& s, float4 inv) {
    const uint32_t oct = (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u) |
                         (inv.w < 0.0f ? 8u : 0u);
    return s.boxes + oct * s.oct_stride;
}

// The traversal stack of one thread for the lean forms (one 8-byte word per entry: reference,
// entry-parameter bits). LocalStack keeps every entry in local memory. SplitStack<S> keeps entries
// [0, S) in shared memory, thread t's in a row of S + 1 words at sm + t * (S + 1) (an odd row
// length: when the lanes of a half-warp stand at the same depth, their 8-byte words fall in
// distinct banks), and entries from S on in local memory. The traversal pushes and pops the same
// entries either way.
struct LocalStack {
    uint2* lm;  // FAST_STACK entries
    __device__ __forceinline__ void put(int i, uint2 e) const { lm[i] = e; }
    __device__ __forceinline__ uint2 get(int i) const { return lm[i]; }
    __device__ __forceinline__ void put_ref(int i, uint32_t r) const { lm[i].x = r; }
    __device__ __forceinline__ uint32_t get_ref(int i) const { return lm[i].x; }
};
template <int S>
struct SplitStack {
    static constexpr int ROW = S + 1;  // words per thread in shared memory (S used)
    uint2* sm;                         // this thread's row in shared memory
    uint2* lm;                         // FAST_STACK entries in local memory (entries below S unused)
    __device__ __forceinline__ void put(int i, uint2 e) const {
        if (i < S) sm[i] = e;
        else lm[i] = e;
    }
    __device__ __forceinline__ uint2 get(int i) const { return i < S ? sm[i] : lm[i]; }
    __device__ __forceinline__ void put_ref(int i, uint32_t r) const {
        if (i < S) sm[i].x = r;
        else lm[i].x = r;
    }
    __device__ __forceinline__ uint32_t get_ref(int i) const { return i < S ? sm[i].x : lm[i].x; }
};

// Closest hit from node `cur` (the root, already tested against the ray). Returns the slot or
// -1; `t_max` ends as the closest hit's parameter.
//
// Loop shape: one iteration is one node visit or one tetrahedron test, so the lanes of a warp at
// a node advance by a node for each tetrahedron the lanes at a leaf test, instead of waiting for
// the longest leaf of the warp. A leaf in progress is its packed reference with the tested
// primitives taken off the front. Each ray's own sequence of node visits and tests, and so its
// result, is the same.
// The top levels of the tree staged in shared memory: wide nodes [0, n) with their (min, max)
// boxes and packed references.
struct TopStage {
    const float4* boxes;
    const uint2* refs;
    uint32_t n;
};

// OCT: the scene has the 16 sign-octant box copies (else the compact layout, one (min, max)
// copy). TOP: nodes below top.n are read from the shared-memory stage.
template <bool COUNT, bool OCT, bool TOP, class Stack>
__device__ __forceinline__ int closest_lean(const WideScene& s, uint32_t cur, float4 no, float4 d, float4 inv, float t_min,
                                            float& t_max, GeomHit& best, const Stack& st, uint32_t* err, Work& work,
                                            const TopStage& top) {
    const float4* ob = OCT ? octant_boxes(s, inv) : s.boxes;
    int slot = -1, sp = 0;
    uint32_t visits = 0;
    // The largest float below t_max (t_max > t_min > 0): with it as the exit bound, exit >= entry
    // holds exactly when exit >= entry and entry < t_max do with t_max, so a child's hit test is
    // one comparison.
    float t_below = __uint_as_float(__float_as_uint(t_max) - 1u);
    if (COUNT && (cur & REF_LEAF)) ++work.leaves;
    // Only node visits are counted against the bound: a leaf's tests end with its count, leaves
    // are entered from node visits or from stack entries, and entries are pushed by node visits.
    for (;;) {
        if (cur & REF_LEAF) {
            const uint32_t k = cur & REF_FIRST_MASK;
            if (COUNT) ++work.tets;
            GeomHit gh;
            if (intersect_lean(s.geoms + 5u * k, no, d, t_min, t_max, &gh)) {
                t_max = gh.lambda;
                t_below = __uint_as_float(__float_as_uint(t_max) - 1u);
                best = gh;
                slot = (int)k;
            }
            cur += REF_NEXT_PRIM;
            if (cur & REF_COUNT_MASK) continue;
        } else {
            if (++visits > MAX_VISITS_FAST) {
                atomicOr(err, ERR_TRAVERSAL_LIMIT);
                break;
            }
            if (COUNT) ++work.nodes;
            float enl, exl, enr, exr;
            uint2 r;
            if (TOP && cur < top.n) {  // a staged node: (min, max) boxes in shared memory
                const float4* b = top.boxes + 4u * cur;
                r = top.refs[cur];
                slab_interval(b[0], b[1], no, inv, t_min, t_below, &enl, &exl);
                slab_interval(b[2], b[3], no, inv, t_min, t_below, &enr, &exr);
            } else {
                const float4* b = ob + 4ull * cur;
                const float4 lnear = __ldg(b), lfar = __ldg(b + 1), rnear = __ldg(b + 2), rfar = __ldg(b + 3);
                r = __ldg(s.refs + cur);
                if (OCT) {
                    slab_octant(lnear, lfar, no, inv, t_min, t_below, &enl, &exl);
                    slab_octant(rnear, rfar, no, inv, t_min, t_below, &enr, &exr);
                } else {  // compact layout: (min, max) boxes
                    slab_interval(lnear, lfar, no, inv, t_min, t_below, &enl, &exl);
                    slab_interval(rnear, rfar, no, inv, t_min, t_below, &enr, &exr);
                }
            }
            const bool hl = exl >= enl;  // and enl < t_max
            const bool hr = exr >= enr;
            if (hl && hr) {
                const bool ln = enl <= enr;
                if (sp < FAST_STACK) st.put(sp++, ln ? make_uint2(r.y, __float_as_uint(enr)) : make_uint2(r.x, __float_as_uint(enl)));
                else atomicOr(err, ERR_BAD_INDEX);
                cur = ln ? r.x : r.y;
                if (COUNT && (cur & REF_LEAF)) ++work.leaves;
                continue;
            }
            if (hl || hr) {
                cur = hl ? r.x : r.y;
                if (COUNT && (cur & REF_LEAF)) ++work.leaves;
                continue;
            }
        }
        bool found = false;
        while (sp > 0) {
            const uint2 e = st.get(--sp);
            if (__uint_as_float(e.y) < t_max) {
                cur = e.x;
                if (COUNT && (cur & REF_LEAF)) ++work.leaves;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return slot;
}

// Any hit in (t_min, t_max) from node `cur` (the root, already tested): left before right, no
// culling (Bvh4D::is_occluded, bvh4d.rs:523-578). (The answer does not depend on the order;
// nearer-first measured 7% slower on the 7.9M-tet scene.)
template <bool COUNT, bool OCT, bool TOP, class Stack>
__device__ __forceinline__ bool any_lean(const WideScene& s, uint32_t cur, float4 no, float4 d, float4 inv, float t_min,
                                         float t_max, const Stack& st, uint32_t* err, Work& work, const TopStage& top) {
    const float4* ob = OCT ? octant_boxes(s, inv) : s.boxes;
    int sp = 0;
    uint32_t visits = 0;
    if (COUNT && (cur & REF_LEAF)) ++work.leaves;
    for (;;) {  // node visits are counted against the bound (see closest_lean)
        if (cur & REF_LEAF) {
            if (COUNT) ++work.tets;
            GeomHit gh;
            if (intersect_lean(s.geoms + 5u * (cur & REF_FIRST_MASK), no, d, t_min, t_max, &gh)) return true;
            cur += REF_NEXT_PRIM;
            if (cur & REF_COUNT_MASK) continue;
        } else {
            if (++visits > MAX_VISITS_FAST) {
                atomicOr(err, ERR_TRAVERSAL_LIMIT);
                return false;
            }
            if (COUNT) ++work.nodes;
            float enl, exl, enr, exr;
            uint2 r;
            if (TOP && cur < top.n) {
                const float4* b = top.boxes + 4u * cur;
                r = top.refs[cur];
                slab_interval(b[0], b[1], no, inv, t_min, t_max, &enl, &exl);
                slab_interval(b[2], b[3], no, inv, t_min, t_max, &enr, &exr);
            } else {
                const float4* b = ob + 4ull * cur;
                const float4 lnear = __ldg(b), lfar = __ldg(b + 1), rnear = __ldg(b + 2), rfar = __ldg(b + 3);
                r = __ldg(s.refs + cur);
                if (OCT) {
                    slab_octant(lnear, lfar, no, inv, t_min, t_max, &enl, &exl);
                    slab_octant(rnear, rfar, no, inv, t_min, t_max, &enr, &exr);
                } else {
                    slab_interval(lnear, lfar, no, inv, t_min, t_max, &enl, &exl);
                    slab_interval(rnear, rfar, no, inv, t_min, t_max, &enr, &exr);
                }
            }
            const bool hl = exl >= enl, hr = exr >= enr;
            if (hl && hr) {
                if (sp < FAST_STACK) st.put_ref(sp++, r.y);
                else atomicOr(err, ERR_BAD_INDEX);
                cur = r.x;
                if (COUNT && (cur & REF_LEAF)) ++work.leaves;
                continue;
            }
            if (hl || hr) {
                cur = hl ? r.x : r.y;
                if (COUNT && (cur & REF_LEAF)) ++work.leaves;
                continue;
            }
        }
        if (sp == 0) return false;
        cur = st.get_ref(--sp);
        if (COUNT && (cur & REF_LEAF)) ++work.leaves;
    }
}

// ---------------------------------------------------------------------------------------------
// Packet traversal: the closest-hit queries of a warp's 32 lanes (the primary rays of one tile of
// neighbouring pixels) walked as one. The warp steps through one node sequence. At an internal node
// every lane that takes part tests both child boxes against its own ray, bounded by its own
// closest hit so far; a child is entered when some lane enters it, and when lanes enter both, the
// child that more of them enter first goes first (the left one on a tie), the other pushed with each
// lane's entry parameter (+inf where the lane misses it) and taken again when some lane still
// enters it before its closest hit. At a leaf every lane that takes part tests the records in
// order. Rays of neighbouring pixels walk nearly the same nodes (on the 7.9M-tet workload the union
// of a 4x8 tile's node visits is 6% above one ray's), so the warp runs one instruction stream with
// warp-wide loads of one node or record, where the per-lane order runs the node and record code
// side by side over lanes standing at different nodes.
//
// The result of each lane is closest_lean's. The closest hit so far is never nearer than the
// reference's final one, so no box the reference enters on the way to its hit is culled, and that
// hit is tested; no nearer hit exists among the records tested; of hits at equal lambda the lane
// keeps the one the reference's near-first order meets first (packet_precedes). This holds as long
// as every hit lies beyond the entry parameter of its leaf's box as computed. A hit's event passes
// the barycentric test, so it lies inside the record's box, which the build pads by 1e-4: in ray
// parameter a margin of 1e-4 / |d| on the entering axis, against a rounding of the computed entry
// of order 1e-7 lambda; only hits far along a fast axis (lambda ~ 100 or more with |d| ~ 8) bring
// the two within a factor of two.
// ---------------------------------------------------------------------------------------------

// Whether hot record a comes before hot record b in the reference's visiting order for this ray
// (a != b): at their lowest common ancestor the near child (smaller entry parameter, the left one on
// equal entries) is entered first; within one leaf, records in index order.
template <bool OCT>
__device__ __noinline__ bool packet_precedes(const WideScene& s, uint32_t a, uint32_t b, float4 no, float4 inv, float t_min,
                                             uint32_t* err) {
    if (s.root_ref & REF_LEAF) return a < b;
    const uint32_t pa = __ldg(s.leafpar + a), pb = __ldg(s.leafpar + b);
    if (pa == pb) return a < b;
    constexpr uint32_t NODE = 0x7FFFFFFFu;
    uint32_t na = pa & NODE, nb = pb & NODE, sa = pa >> 31, sb = pb >> 31;
    uint32_t da = 0, db = 0;
    for (uint32_t w = na; da <= FAST_MAX_DEPTH; ++da) {
        const uint32_t u = __ldg(s.up + w);
        if (u == ~0u) break;
        w = u & NODE;
    }
    for (uint32_t w = nb; db <= FAST_MAX_DEPTH; ++db) {
        const uint32_t u = __ldg(s.up + w);
        if (u == ~0u) break;
        w = u & NODE;
    }
    if (da > FAST_MAX_DEPTH || db > FAST_MAX_DEPTH) {
        atomicOr(err, ERR_BAD_INDEX);
        return a < b;
    }
    // Climb to equal depth, then together to the first common node; (n, s): the branch towards the
    // record is child s of node n.
    for (; da > db; --da) {
        const uint32_t u = __ldg(s.up + na);
        sa = u >> 31;
        na = u & NODE;
    }
    for (; db > da; --db) {
        const uint32_t u = __ldg(s.up + nb);
        sb = u >> 31;
        nb = u & NODE;
    }
    for (; na != nb; --da) {
        if (da == 0) {
            atomicOr(err, ERR_BAD_INDEX);
            return a < b;
        }
        const uint32_t ua = __ldg(s.up + na), ub = __ldg(s.up + nb);
        sa = ua >> 31;
        na = ua & NODE;
        sb = ub >> 31;
        nb = ub & NODE;
    }
    const float4* bx = (OCT ? octant_boxes(s, inv) : s.boxes) + 4ull * na;
    const float4 b0 = __ldg(bx), b1 = __ldg(bx + 1), b2 = __ldg(bx + 2), b3 = __ldg(bx + 3);
    const float big = 3.0e38f;  // the entry parameters do not depend on the exit bound
    float enl, exl, enr, exr;
    if (OCT) {
        slab_octant(b0, b1, no, inv, t_min, big, &enl, &exl);
        slab_octant(b2, b3, no, inv, t_min, big, &enr, &exr);
    } else {
        slab_interval(b0, b1, no, inv, t_min, big, &enl, &exl);
        slab_interval(b2, b3, no, inv, t_min, big, &enr, &exr);
    }
    const bool left_first = enl <= enr;
    return sa == 0 ? left_first : !left_first;
}

// The packet form of closest_lean for the whole warp (all 32 lanes call it together, converged).
// `in`: this lane's ray enters the scene's box (the others take no part). Returns the slot or -1;
// `t_max` ends as the closest hit's parameter.
template <bool OCT, class Stack>
__device__ __forceinline__ int closest_packet(const WideScene& s, bool in, float4 no, float4 d, float4 inv, float t_min,
                                              float& t_max, GeomHit& best, const Stack& st, uint32_t* err) {
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const float none = __uint_as_float(0x7F800000u);  // +inf: the lane does not enter the pushed child
    const float4* ob = OCT ? octant_boxes(s, inv) : s.boxes;
    int slot = -1, sp = 0;
    uint32_t visits = 0;
    float t_below = __uint_as_float(__float_as_uint(t_max) - 1u);
    uint32_t cur = s.root_ref;
    for (;;) {
        if (cur & REF_LEAF) {
            const uint32_t k = cur & REF_FIRST_MASK;
            if (in) {
                GeomHit gh;
                // Hits up to and including t_max, so that a hit at the closest hit's lambda is seen.
                if (intersect_lean(s.geoms + 5u * k, no, d, t_min, __uint_as_float(__float_as_uint(t_max) + 1u), &gh)) {
                    if (gh.lambda < t_max) {
                        t_max = gh.lambda;
                        t_below = __uint_as_float(__float_as_uint(t_max) - 1u);
                        best = gh;
                        slot = (int)k;
                    } else if (slot >= 0 && packet_precedes<OCT>(s, k, (uint32_t)slot, no, inv, t_min, err)) {
                        best = gh;
                        slot = (int)k;
                    }
                }
            }
            cur += REF_NEXT_PRIM;
            if (cur & REF_COUNT_MASK) continue;
        } else {
            if (++visits > MAX_VISITS_FAST) {
                atomicOr(err, ERR_TRAVERSAL_LIMIT);
                break;
            }
            const uint2 r = __ldg(s.refs + cur);
            // Every lane computes (the warp runs the code once either way); lanes that take no part
            // are masked out, so the step has no divergent branch.
            const float4* b = ob + 4ull * cur;
            const float4 lnear = __ldg(b), lfar = __ldg(b + 1), rnear = __ldg(b + 2), rfar = __ldg(b + 3);
            float enl, exl, enr, exr;
            if (OCT) {
                slab_octant(lnear, lfar, no, inv, t_min, t_below, &enl, &exl);
                slab_octant(rnear, rfar, no, inv, t_min, t_below, &enr, &exr);
            } else {
                slab_interval(lnear, lfar, no, inv, t_min, t_below, &enl, &exl);
                slab_interval(rnear, rfar, no, inv, t_min, t_below, &enr, &exr);
            }
            const bool hl = in && exl >= enl;  // and enl < t_max
            const bool hr = in && exr >= enr;
            const uint32_t ml = __ballot_sync(FULL, hl), mr = __ballot_sync(FULL, hr);
            if (ml && mr) {
                const uint32_t nl = __popc(__ballot_sync(FULL, hl && (!hr || enl <= enr)));
                const bool left_first = 2u * nl >= (uint32_t)__popc(ml | mr);
                if (sp < FAST_STACK)
                    st.put(sp++, left_first ? make_uint2(r.y, __float_as_uint(hr ? enr : none))
                                            : make_uint2(r.x, __float_as_uint(hl ? enl : none)));
                else atomicOr(err, ERR_BAD_INDEX);
                cur = left_first ? r.x : r.y;
                in = left_first ? hl : hr;
                continue;
            }
            if (ml | mr) {
                cur = ml ? r.x : r.y;
                in = ml ? hl : hr;
                continue;
            }
        }
        bool found = false;
        while (sp > 0) {
            const uint2 e = st.get(--sp);
            const bool take = __uint_as_float(e.y) < t_max;
            if (__any_sync(FULL, take)) {
                cur = e.x;
                in = take;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return slot;
}

// The packet form of any_lean for the whole warp (all 32 lanes call it together, converged): the
// lanes' any-hit queries walked as one node sequence, left child first. A lane takes part in a
// node or leaf its own ray enters, and stops once it has a hit; the walk ends when no lane still
// searching takes part in anything left. Every lane tests records of leaves its ray enters until
// one hits, so its answer is any_lean's (an any-hit answer does not depend on the order).
// `in`: this lane has a query whose ray enters the scene's box.
template <bool OCT, class Stack>
__device__ __forceinline__ bool any_packet(const WideScene& s, bool in, float4 no, float4 d, float4 inv, float t_min,
                                           float t_max, const Stack& st, uint32_t* err) {
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const float4* ob = OCT ? octant_boxes(s, inv) : s.boxes;
    bool hit = false, part = in;
    int sp = 0;
    uint32_t visits = 0;
    uint32_t cur = s.root_ref;
    for (;;) {
        if (cur & REF_LEAF) {
            if (part && !hit) {
                GeomHit gh;
                hit = intersect_lean(s.geoms + 5u * (cur & REF_FIRST_MASK), no, d, t_min, t_max, &gh);
            }
            cur += REF_NEXT_PRIM;
            if ((cur & REF_COUNT_MASK) && __any_sync(FULL, part && !hit)) continue;
        } else {
            if (++visits > MAX_VISITS_FAST) {
                atomicOr(err, ERR_TRAVERSAL_LIMIT);
                break;
            }
            const uint2 r = __ldg(s.refs + cur);
            const float4* b = ob + 4ull * cur;
            const float4 lnear = __ldg(b), lfar = __ldg(b + 1), rnear = __ldg(b + 2), rfar = __ldg(b + 3);
            float enl, exl, enr, exr;
            if (OCT) {
                slab_octant(lnear, lfar, no, inv, t_min, t_max, &enl, &exl);
                slab_octant(rnear, rfar, no, inv, t_min, t_max, &enr, &exr);
            } else {
                slab_interval(lnear, lfar, no, inv, t_min, t_max, &enl, &exl);
                slab_interval(rnear, rfar, no, inv, t_min, t_max, &enr, &exr);
            }
            const bool live = part && !hit;
            const bool hl = live && exl >= enl, hr = live && exr >= enr;
            const uint32_t ml = __ballot_sync(FULL, hl), mr = __ballot_sync(FULL, hr);
            if (ml && mr) {
                if (sp < FAST_STACK) st.put(sp++, make_uint2(r.y, hr ? 1u : 0u));
                else atomicOr(err, ERR_BAD_INDEX);
                cur = r.x;
                part = hl;
                continue;
            }
            if (ml | mr) {
                cur = ml ? r.x : r.y;
                part = ml ? hl : hr;
                continue;
            }
        }
        bool found = false;
        while (sp > 0) {
            const uint2 e = st.get(--sp);
            const bool take = e.y != 0u && !hit;
            if (__any_sync(FULL, take)) {
                cur = e.x;
                part = take;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return hit;
}

}  // namespace srk
