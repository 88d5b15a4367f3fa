// BVH build on the GPU: the reference's Bvh4D::build (bvh4d.rs:123-141, 287-427) over simplex
// boxes given in build order, producing the same node array (depth-first, left child next) and the
// same leaf order as the serial build:
//   - node bounds and centroid bounds are unions of the primitives' boxes and centroids (min / max
//     are exact, so any reduction order gives the same floats; boxes carry the builder's 1e-4
//     padding, so no coordinate is -0 and ordered-integer atomics give fmin/fmax's values);
//   - split: 8 bins on each of the four axes whose centroid extent is >= 1e-4, bin index
//     min(trunc((c - min) * (8 / extent)), 7), the SAH cost count * box_measure for the left and
//     right prefixes, the first strictly lower cost in axis order 0..3 and bin order 6..0; with no
//     valid bin split, the centroid box's centre on its longest axis (a leaf below 1e-5);
//   - partition: the reference's in-place pass (elements left of the split swapped to the front in
//     order). Its result: the left elements in their order, then the right elements in the order of
//     a queue that receives each right element and rotates by one at every left element that finds
//     it non-empty. Large nodes compute that order in parallel (prefix sums, then the queue's
//     contents by pointer jumping); small subtrees run the pass itself;
//   - a split that leaves one side empty falls back in the reference to a selection by median
//     (nth_element); the build reports that case as unsupported instead (no synthetic scene of the
//     configurations reaches it).
// Large nodes (more than SMALL primitives) are split level by level across the whole GPU; each
// subtree of at most SMALL primitives is built by one block in shared memory, depth first. The host
// joins the parts in depth-first order (it sees only the few thousand large nodes).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "sr_build.h"

namespace srk {

namespace {

constexpr uint32_t SMALL = 2048;       // primitives of a subtree built by one block
constexpr uint32_t CHUNK = 2048;       // positions per block in the large-node reductions
constexpr int BINS = 8;

// Floats as integers whose order is the floats' order (min / max by integer atomics).
__device__ __forceinline__ int okey(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float oval(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }
inline float oval_host(int k) {
    const int i = k >= 0 ? k : k ^ 0x7FFFFFFF;
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}
__device__ __forceinline__ float ax(float4 v, int a) { return a == 0 ? v.x : a == 1 ? v.y : a == 2 ? v.z : v.w; }

// box_measure (bvh4d.rs:8-13) with e = hi - lo in (t, x, y, z) order.
__device__ __forceinline__ float box_measure(const float* lo, const float* hi) {
    const float et = hi[0] - lo[0], ex = hi[1] - lo[1], ey = hi[2] - lo[2], ez = hi[3] - lo[3];
    return ex * ey + ey * ez + ez * ex + 0.22f * et * (ex + ey + ez);
}

// The split decision of one node from its centroid bounds and bins (min / max as ordered
// integers, counts). Returns 0 for a split (axis, pos), 1 for a leaf.
__device__ int decide_split(const int* clo, const int* chi, const int (*blo)[4], const int (*bhi)[4], const uint32_t* bcnt,
                            int* axis_out, float* pos_out) {
    float ext[4], amin[4];
    bool live[4];
    for (int a = 0; a < 4; ++a) {
        amin[a] = oval(clo[a]);
        ext[a] = oval(chi[a]) - amin[a];
        live[a] = ext[a] >= 1e-4f;
    }
    int best_axis = 0;
    float best_pos = 0.0f, best_cost = INFINITY;
    for (int a = 0; a < 4; ++a) {
        if (!live[a]) continue;
        float lbl[7][4], lbh[7][4];
        uint32_t lc[7], cc = 0;
        float cl[4] = {INFINITY, INFINITY, INFINITY, INFINITY}, ch[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (int i = 0; i < 7; ++i) {
            const int b = a * BINS + i;
            for (int k = 0; k < 4; ++k) { cl[k] = fminf(cl[k], oval(blo[b][k])); ch[k] = fmaxf(ch[k], oval(bhi[b][k])); }
            cc += bcnt[b];
            for (int k = 0; k < 4; ++k) { lbl[i][k] = cl[k]; lbh[i][k] = ch[k]; }
            lc[i] = cc;
        }
        float rl[4] = {INFINITY, INFINITY, INFINITY, INFINITY}, rh[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
        uint32_t rc = 0;
        for (int i = 6; i >= 0; --i) {
            const int b = a * BINS + i + 1;
            for (int k = 0; k < 4; ++k) { rl[k] = fminf(rl[k], oval(blo[b][k])); rh[k] = fmaxf(rh[k], oval(bhi[b][k])); }
            rc += bcnt[b];
            if (lc[i] > 0 && rc > 0) {
                const float cost = (float)lc[i] * box_measure(lbl[i], lbh[i]) + (float)rc * box_measure(rl, rh);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_pos = amin[a] + ((float)(i + 1) / 8.0f) * ext[a];
                }
            }
        }
    }
    if (best_cost == INFINITY) {
        float me = -1.0f;
        for (int a = 0; a < 4; ++a)
            if (ext[a] > me) { me = ext[a]; best_axis = a; }
        if (me < 1e-5f) return 1;
        best_pos = (oval(clo[best_axis]) + oval(chi[best_axis])) * 0.5f;
    }
    *axis_out = best_axis;
    *pos_out = best_pos;
    return 0;
}

// decide_split computed by the 32 lanes of a warp, lane 8a + i holding bin i of axis a: the left
// unions and counts of bins 0..i and the right ones of bins i+1..7 by segmented scans (min / max
// and integer sums are exact in any order), then each candidate's cost by the same expression, and
// the first strictly lowest cost in the serial order (axis 0..3, split 6..0) by a reduction whose
// ties go to the earlier candidate. Every lane returns the decision.
struct SplitChoice {
    int leaf, axis;
    float pos;
};
__device__ SplitChoice decide_split_warp(const int* clo, const int* chi, const int (*blo)[4], const int (*bhi)[4],
                                         const uint32_t* bcnt, uint32_t lane) {
    const int a = (int)(lane >> 3), i = (int)(lane & 7u);
    const float amin = oval(clo[a]);
    const float ext = oval(chi[a]) - amin;
    const bool live = ext >= 1e-4f;
    float l[8], r[8];
    for (int k = 0; k < 4; ++k) {
        l[k] = oval(blo[lane][k]);
        l[4 + k] = oval(bhi[lane][k]);
    }
    uint32_t lc = bcnt[lane];
    for (int k = 0; k < 8; ++k) r[k] = l[k];
    uint32_t rc = lc;
    for (int d = 1; d < 8; d <<= 1) {  // inclusive scans within the axis's 8 lanes
        uint32_t up_c = __shfl_up_sync(0xFFFFFFFFu, lc, d, 8), dn_c = __shfl_down_sync(0xFFFFFFFFu, rc, d, 8);
        for (int k = 0; k < 8; ++k) {
            const float u = __shfl_up_sync(0xFFFFFFFFu, l[k], d, 8), v = __shfl_down_sync(0xFFFFFFFFu, r[k], d, 8);
            if (i >= d) l[k] = k < 4 ? fminf(l[k], u) : fmaxf(l[k], u);
            if (i + d < 8) r[k] = k < 4 ? fminf(r[k], v) : fmaxf(r[k], v);
        }
        if (i >= d) lc += up_c;
        if (i + d < 8) rc += dn_c;
    }
    // The right side of split i is bins i+1..7: the next lane's suffix.
    float rr[8];
    for (int k = 0; k < 8; ++k) rr[k] = __shfl_down_sync(0xFFFFFFFFu, r[k], 1, 8);
    const uint32_t rrc = __shfl_down_sync(0xFFFFFFFFu, rc, 1, 8);
    float cost = INFINITY;
    if (live && i < 7 && lc > 0 && rrc > 0)
        cost = (float)lc * box_measure(l, l + 4) + (float)rrc * box_measure(rr, rr + 4);
    int order = (cost < INFINITY) ? a * 8 + (6 - i) : 1 << 20;  // the serial loop's visiting order
    if (!(cost < INFINITY)) cost = INFINITY;
    for (int off = 16; off > 0; off >>= 1) {
        const float oc = __shfl_xor_sync(0xFFFFFFFFu, cost, off);
        const int oo = __shfl_xor_sync(0xFFFFFFFFu, order, off);
        if (oc < cost || (oc == cost && oo < order)) {
            cost = oc;
            order = oo;
        }
    }
    SplitChoice c{0, 0, 0.0f};
    if (cost < INFINITY) {
        const int ba = order >> 3, bi = 6 - (order & 7);
        const float bmin = oval(clo[ba]), bext = oval(chi[ba]) - bmin;
        c.axis = ba;
        c.pos = bmin + ((float)(bi + 1) / 8.0f) * bext;
        return c;
    }
    float me = -1.0f;
    for (int x = 0; x < 4; ++x) {
        const float e = oval(chi[x]) - oval(clo[x]);
        if (e > me) { me = e; c.axis = x; }
    }
    if (me < 1e-5f) { c.leaf = 1; return c; }
    c.pos = (oval(clo[c.axis]) + oval(chi[c.axis])) * 0.5f;
    return c;
}

// Bin of centroid coordinate c: min(trunc((c - amin) * inv), 7), 0 for NaN or <= 0.
__device__ __forceinline__ int bin_of(float c, float amin, float inv) {
    const float x = (c - amin) * inv;
    if (!(x > 0.0f)) return 0;
    return x >= 7.0f ? 7 : (int)x;
}

// ---------------------------------------------------------------------------------------------
// Large nodes, one level at a time.
// ---------------------------------------------------------------------------------------------
struct LTask {
    uint32_t start, count, qbase;
};
struct LHead {  // per large node of the level; read back by the host
    int blo[4], bhi[4], clo[4], chi[4];
    int leaf, axis;
    float pos;
    uint32_t m, S;
};
struct LBins {
    int lo[32][4], hi[32][4];
    uint32_t cnt[32];
};
struct Chunk {
    uint32_t task, q0, q1;  // compacted positions [q0, q1) of `task`
};

__global__ void k_init_build(const float4* box, uint32_t n, float4* cen, uint32_t* perm) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = box[2ull * i], b = box[2ull * i + 1];
    cen[i] = make_float4((a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f, (a.w + b.w) * 0.5f);
    perm[i] = i;
}

__global__ void k_init_heads(LHead* h, LBins* b, uint32_t nt) {
    uint32_t t = blockIdx.x;
    if (t >= nt) return;
    for (uint32_t j = threadIdx.x; j < 16; j += blockDim.x) {
        int* v = &h[t].blo[0];
        v[j] = (j / 4) % 2 == 0 ? okey(INFINITY) : okey(-INFINITY);
    }
    for (uint32_t j = threadIdx.x; j < 32 * 4; j += blockDim.x) {
        (&b[t].lo[0][0])[j] = okey(INFINITY);
        (&b[t].hi[0][0])[j] = okey(-INFINITY);
    }
    for (uint32_t j = threadIdx.x; j < 32; j += blockDim.x) b[t].cnt[j] = 0;
    if (threadIdx.x == 0) { h[t].leaf = 0; h[t].m = 0; h[t].S = 0; }
}

// Bounds of each chunk, merged into its node with atomics (block reduction first).
__global__ void __launch_bounds__(256) k_large_bounds(const Chunk* chunks, const LTask* tasks, const uint32_t* perm,
                                                     const float4* box, const float4* cen, LHead* heads) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    float v[16];
    for (int k = 0; k < 4; ++k) { v[k] = INFINITY; v[4 + k] = -INFINITY; v[8 + k] = INFINITY; v[12 + k] = -INFINITY; }
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
        const uint32_t e = perm[t.start + (q - t.qbase)];
        const float4 a = box[2ull * e], b = box[2ull * e + 1], m = cen[e];
        for (int k = 0; k < 4; ++k) {
            v[k] = fminf(v[k], ax(a, k));
            v[4 + k] = fmaxf(v[4 + k], ax(b, k));
            v[8 + k] = fminf(v[8 + k], ax(m, k));
            v[12 + k] = fmaxf(v[12 + k], ax(m, k));
        }
    }
    for (int k = 0; k < 16; ++k) {
        const bool mx = (k / 4) % 2 == 1;
        float x = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            const float y = __shfl_xor_sync(0xFFFFFFFFu, x, o);
            x = mx ? fmaxf(x, y) : fminf(x, y);
        }
        v[k] = x;
    }
    __shared__ float part[8][16];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 16; ++k) part[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < 16) {
        const int k = threadIdx.x;
        const bool mx = (k / 4) % 2 == 1;
        float x = part[0][k];
        for (int j = 1; j < (int)(blockDim.x >> 5); ++j) x = mx ? fmaxf(x, part[j][k]) : fminf(x, part[j][k]);
        int* dst = &heads[c.task].blo[0];
        if (mx) atomicMax(dst + k, okey(x));
        else atomicMin(dst + k, okey(x));
    }
}

// Bins of each chunk (shared-memory atomics), merged into its node's bins.
__global__ void __launch_bounds__(256) k_large_bins(const Chunk* chunks, const LTask* tasks, const uint32_t* perm,
                                                   const float4* box, const float4* cen, const LHead* heads,
                                                   LBins* bins) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    __shared__ int slo[32][4], shi[32][4];
    __shared__ uint32_t scnt[32];
    __shared__ float amin[4], inv[4];
    __shared__ int live[4];
    for (uint32_t j = threadIdx.x; j < 128; j += blockDim.x) { (&slo[0][0])[j] = okey(INFINITY); (&shi[0][0])[j] = okey(-INFINITY); }
    if (threadIdx.x < 32) scnt[threadIdx.x] = 0;
    if (threadIdx.x < 4) {
        const int a = threadIdx.x;
        const float mn = oval(heads[c.task].clo[a]), ext = oval(heads[c.task].chi[a]) - mn;
        amin[a] = mn;
        inv[a] = 8.0f / ext;
        live[a] = ext >= 1e-4f;
    }
    __syncthreads();
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
        const uint32_t e = perm[t.start + (q - t.qbase)];
        const float4 a = box[2ull * e], b = box[2ull * e + 1], m = cen[e];
        for (int x = 0; x < 4; ++x) {
            if (!live[x]) continue;
            const int bi = x * BINS + bin_of(ax(m, x), amin[x], inv[x]);
            for (int k = 0; k < 4; ++k) {
                atomicMin(&slo[bi][k], okey(ax(a, k)));
                atomicMax(&shi[bi][k], okey(ax(b, k)));
            }
            atomicAdd(&scnt[bi], 1u);
        }
    }
    __syncthreads();
    LBins& g = bins[c.task];
    for (uint32_t j = threadIdx.x; j < 32; j += blockDim.x) {
        if (scnt[j] == 0) continue;
        atomicAdd(&g.cnt[j], scnt[j]);
        for (int k = 0; k < 4; ++k) {
            atomicMin(&g.lo[j][k], slo[j][k]);
            atomicMax(&g.hi[j][k], shi[j][k]);
        }
    }
}

__global__ void k_large_decide(LHead* heads, const LBins* bins, uint32_t nt) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int axis = 0;
    float pos = 0.0f;
    heads[t].leaf = decide_split(heads[t].clo, heads[t].chi, bins[t].lo, bins[t].hi, bins[t].cnt, &axis, &pos);
    heads[t].axis = axis;
    heads[t].pos = pos;
}

// Per compacted position: the left flag, and the node id as the scan key.
__global__ void k_large_flags(const Chunk* chunks, const LTask* tasks, const LHead* heads, const uint32_t* perm,
                              const float4* cen, uint32_t* flag, uint32_t* key) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    const LHead& h = heads[c.task];
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
        key[q] = c.task;
        flag[q] = h.leaf ? 0u : (ax(cen[perm[t.start + (q - t.qbase)]], h.axis) < h.pos ? 1u : 0u);
    }
}

// From the left counts before each position: the service flag (a left element that finds the
// queue non-empty).
__global__ void k_large_service(const Chunk* chunks, const LTask* tasks, const uint32_t* flag, const uint32_t* lb,
                                uint32_t* svc) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
        const uint32_t rb = (q - t.qbase) - lb[q];
        svc[q] = (flag[q] && rb > 0) ? 1u : 0u;
    }
}

// The queue's enqueue list: a right element at enqueue index rb + sb; a service event re-enqueues
// the sb-th enqueued element (items >= 0 are resolved, refs point into the same list).
__global__ void k_large_events(const Chunk* chunks, const LTask* tasks, const uint32_t* perm, const uint32_t* flag,
                               const uint32_t* lb, const uint32_t* svc, const uint32_t* sb, int* eitem, int* eref,
                               LHead* heads) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    const uint32_t ebase = 2u * t.qbase;
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
        const uint32_t i = q - t.qbase, rb = i - lb[q];
        const uint32_t e = ebase + rb + sb[q];
        if (!flag[q]) {
            eitem[e] = (int)perm[t.start + i];
        } else if (svc[q]) {
            eref[e] = (int)(ebase + sb[q]);
        }
        if (i == t.count - 1) {
            heads[c.task].m = lb[q] + flag[q];
            heads[c.task].S = sb[q] + svc[q];
        }
    }
}

// One round of pointer jumping over the enqueue list (reads a, writes b).
__global__ void k_jump(const int* item_a, const int* ref_a, int* item_b, int* ref_b, uint32_t len) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= len) return;
    int it = item_a[j], rf = ref_a[j];
    if (it < 0 && rf >= 0) {
        const int it2 = item_a[rf];
        if (it2 >= 0) {
            it = it2;
            rf = -1;
        } else {
            rf = ref_a[rf];
        }
    }
    item_b[j] = it;
    ref_b[j] = rf;
}

// The partitioned order: left elements at their left rank, then the queue's final contents.
__global__ void k_large_scatter(const Chunk* chunks, const LTask* tasks, const LHead* heads, const uint32_t* perm,
                                const uint32_t* flag, const uint32_t* lb, const int* eitem, uint32_t* perm_out) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    const LHead& h = heads[c.task];
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
        const uint32_t i = q - t.qbase;
        if (h.leaf) {
            perm_out[t.start + i] = perm[t.start + i];
            continue;
        }
        if (flag[q]) perm_out[t.start + lb[q]] = perm[t.start + i];
        if (i >= h.m) perm_out[t.start + i] = (uint32_t)eitem[2u * t.qbase + h.S + (i - h.m)];
    }
}

__global__ void k_copy_range(const Chunk* chunks, const LTask* tasks, const uint32_t* src, uint32_t* dst) {
    const Chunk c = chunks[blockIdx.x];
    const LTask t = tasks[c.task];
    for (uint32_t q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) dst[t.start + (q - t.qbase)] = src[t.start + (q - t.qbase)];
}

// ---------------------------------------------------------------------------------------------
// Small subtrees: one block builds the subtree of one node depth first in shared memory, as the
// serial build does. Nodes go to `out + 2 * start` with links relative to the subtree's root.
// ---------------------------------------------------------------------------------------------
struct STask {
    uint32_t start, count;
};
struct SResult {
    uint32_t nodes, depth, max_leaf, bad;
};

__global__ void __launch_bounds__(256) k_small_build(const STask* tasks, const uint32_t* ids, const float4* box,
                                                    const float4* cen, uint32_t* perm, SrGpuNode* out, SResult* res) {
    extern __shared__ float4 sm[];
    const uint32_t task = ids[blockIdx.x];
    const STask tk = tasks[task];
    const uint32_t n = tk.count;
    float4* slo = sm;
    float4* shi = sm + SMALL;
    float4* scen = sm + 2 * SMALL;
    uint32_t* sidx = reinterpret_cast<uint32_t*>(sm + 3 * SMALL);  // build index of each local element
    uint16_t* ord = reinterpret_cast<uint16_t*>(sidx + SMALL);     // the working order (local ids)
    __shared__ int bl[32][4], bh[32][4];
    __shared__ uint32_t bc[32];
    __shared__ float part[8][16];
    __shared__ int red[16];
    __shared__ uint32_t fs[64], fc[64], fpatch[64], fdepth[64];  // DFS frames
    __shared__ int sp, node_count, cur_leaf, cur_axis, max_depth, max_leaf, bad;
    __shared__ float cur_pos;
    __shared__ uint32_t cur_s, cur_c, cur_patch, cur_depth, cur_mid;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t e = perm[tk.start + i];
        slo[i] = box[2ull * e];
        shi[i] = box[2ull * e + 1];
        scen[i] = cen[e];
        sidx[i] = e;
        ord[i] = (uint16_t)i;
    }
    if (threadIdx.x == 0) {
        sp = 0;
        fs[0] = 0; fc[0] = n; fpatch[0] = 0xFFFFFFFFu; fdepth[0] = 1;
        sp = 1;
        node_count = 0;
        max_depth = 0;
        max_leaf = 0;
        bad = 0;
    }
    __syncthreads();
    SrGpuNode* o = out + 2ull * tk.start;
    while (true) {
        if (threadIdx.x == 0) {
            if (sp > 0) {
                --sp;
                cur_s = fs[sp]; cur_c = fc[sp]; cur_patch = fpatch[sp]; cur_depth = fdepth[sp];
            } else {
                cur_c = 0;
            }
        }
        __syncthreads();
        if (cur_c == 0) break;
        const uint32_t s = cur_s, c = cur_c;
        if (c <= 3) {  // a leaf needs only its box: thread 0 takes the min / max of its few boxes
            if (threadIdx.x == 0) {
                float lo[4] = {INFINITY, INFINITY, INFINITY, INFINITY}, hi[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
                for (uint32_t i = 0; i < c; ++i) {
                    const uint32_t e = ord[s + i];
                    const float4 a = slo[e], b = shi[e];
                    for (int k = 0; k < 4; ++k) { lo[k] = fminf(lo[k], ax(a, k)); hi[k] = fmaxf(hi[k], ax(b, k)); }
                }
                const int idx = node_count++;
                SrGpuNode nd;
                for (int k = 0; k < 4; ++k) { nd.min[k] = lo[k]; nd.max[k] = hi[k]; }
                nd.right_or_first = tk.start + s;
                nd.count = c;
                nd.left = 0;
                nd.pad = 0;
                if ((int)c > max_leaf) max_leaf = (int)c;
                o[idx] = nd;
                if (cur_patch != 0xFFFFFFFFu) o[cur_patch].right_or_first = (uint32_t)idx;
                if ((int)cur_depth > max_depth) max_depth = (int)cur_depth;
            }
            __syncthreads();  // every thread has read this node before the next is popped
            continue;
        }
        // Bounds and centroid bounds.
        float v[16];
        for (int k = 0; k < 4; ++k) { v[k] = INFINITY; v[4 + k] = -INFINITY; v[8 + k] = INFINITY; v[12 + k] = -INFINITY; }
        for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
            const uint32_t e = ord[s + i];
            const float4 a = slo[e], b = shi[e], m = scen[e];
            for (int k = 0; k < 4; ++k) {
                v[k] = fminf(v[k], ax(a, k));
                v[4 + k] = fmaxf(v[4 + k], ax(b, k));
                v[8 + k] = fminf(v[8 + k], ax(m, k));
                v[12 + k] = fmaxf(v[12 + k], ax(m, k));
            }
        }
        for (int k = 0; k < 16; ++k) {
            const bool mx = (k / 4) % 2 == 1;
            float x = v[k];
            for (int off = 16; off > 0; off >>= 1) {
                const float y = __shfl_xor_sync(0xFFFFFFFFu, x, off);
                x = mx ? fmaxf(x, y) : fminf(x, y);
            }
            v[k] = x;
        }
        if ((threadIdx.x & 31) == 0)
            for (int k = 0; k < 16; ++k) part[threadIdx.x >> 5][k] = v[k];
        for (uint32_t j = threadIdx.x; j < 128; j += blockDim.x) { (&bl[0][0])[j] = okey(INFINITY); (&bh[0][0])[j] = okey(-INFINITY); }
        if (threadIdx.x < 32) bc[threadIdx.x] = 0;
        __syncthreads();
        if (threadIdx.x < 16) {
            const int k = threadIdx.x;
            const bool mx = (k / 4) % 2 == 1;
            float x = part[0][k];
            for (int j = 1; j < (int)(blockDim.x >> 5); ++j) x = mx ? fmaxf(x, part[j][k]) : fminf(x, part[j][k]);
            red[k] = okey(x);
        }
        __syncthreads();
        const bool small_leaf = c <= 3;
        if (!small_leaf) {
            // Bins.
            float amin[4], inv[4];
            bool live[4];
            for (int a = 0; a < 4; ++a) {
                amin[a] = oval(red[8 + a]);
                const float ext = oval(red[12 + a]) - amin[a];
                inv[a] = 8.0f / ext;
                live[a] = ext >= 1e-4f;
            }
            for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
                const uint32_t e = ord[s + i];
                const float4 a = slo[e], b = shi[e], m = scen[e];
                for (int x = 0; x < 4; ++x) {
                    if (!live[x]) continue;
                    const int bi = x * BINS + bin_of(ax(m, x), amin[x], inv[x]);
                    for (int k = 0; k < 4; ++k) {
                        atomicMin(&bl[bi][k], okey(ax(a, k)));
                        atomicMax(&bh[bi][k], okey(ax(b, k)));
                    }
                    atomicAdd(&bc[bi], 1u);
                }
            }
            __syncthreads();
        }
        SplitChoice ch{1, 0, 0.0f};
        if (!small_leaf && threadIdx.x < 32) ch = decide_split_warp(red + 8, red + 12, bl, bh, bc, threadIdx.x);
        if (threadIdx.x == 0) {
            int leaf = ch.leaf, axis = ch.axis;
            const float pos = ch.pos;
            uint32_t mid = 0;
            if (!leaf) {
                // The reference's partition pass.
                for (uint32_t i = 0; i < c; ++i) {
                    const uint16_t e = ord[s + i];
                    if (ax(scen[e], axis) < pos) {
                        ord[s + i] = ord[s + mid];
                        ord[s + mid] = e;
                        ++mid;
                    }
                }
                if (mid == 0 || mid == c) {  // the reference selects by median here: not supported
                    bad = 1;
                    leaf = 1;
                }
            }
            const int idx = node_count++;
            SrGpuNode nd;
            for (int k = 0; k < 4; ++k) { nd.min[k] = oval(red[k]); nd.max[k] = oval(red[4 + k]); }
            if (leaf) {
                nd.right_or_first = tk.start + s;
                nd.count = c;
                nd.left = 0;
                if ((int)c > max_leaf) max_leaf = (int)c;
            } else {
                nd.right_or_first = 0;
                nd.count = 0;
                nd.left = (uint32_t)idx + 1;
            }
            nd.pad = 0;
            o[idx] = nd;
            if (cur_patch != 0xFFFFFFFFu) o[cur_patch].right_or_first = (uint32_t)idx;
            if ((int)cur_depth > max_depth) max_depth = (int)cur_depth;
            if (!leaf) {
                if (sp + 2 > 64) {
                    bad = 2;
                } else {
                    // Right pushed first, so the left subtree is built first; its node patches the
                    // parent's right link when it is emitted.
                    fs[sp] = s + mid; fc[sp] = c - mid; fpatch[sp] = (uint32_t)idx; fdepth[sp] = cur_depth + 1; ++sp;
                    fs[sp] = s; fc[sp] = mid; fpatch[sp] = 0xFFFFFFFFu; fdepth[sp] = cur_depth + 1; ++sp;
                }
            }
        }
        __syncthreads();
    }
    // The subtree's leaf order: the build indices in the final local order.
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) perm[tk.start + i] = sidx[ord[i]];
    if (threadIdx.x == 0) res[task] = SResult{(uint32_t)node_count, (uint32_t)max_depth, (uint32_t)max_leaf, (uint32_t)bad};
}

// The same build for subtrees of at most TINY primitives, one warp each (WARPS_TINY per block):
// the same bounds, bins, decision and partition pass with warp synchronisation only, so a launch
// of small chunks lasts about as many warp steps as its largest chunk has nodes.
constexpr uint32_t TINY = 256;
constexpr uint32_t WARPS_TINY = 4;
struct TinyShared {
    float4 lo[TINY], hi[TINY], cen[TINY];
    uint32_t sidx[TINY];
    uint16_t ord[TINY];
    int bl[32][4], bh[32][4];
    uint32_t bc[32];
    int red[16];
    uint32_t fs[64], fc[64], fpatch[64], fdepth[64];
    uint32_t cur_s, cur_c, cur_patch, cur_depth;
    int sp, node_count, max_depth, max_leaf, bad;
};

__global__ void __launch_bounds__(32 * WARPS_TINY) k_small_build_warp(const STask* tasks, const uint32_t* ids,
                                                                      uint32_t n_ids, const float4* box,
                                                                      const float4* cen, uint32_t* perm, SrGpuNode* out,
                                                                      SResult* res) {
    extern __shared__ float4 smw[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t slot = blockIdx.x * WARPS_TINY + warp;
    if (slot >= n_ids) return;  // whole warps leave together
    TinyShared& w = reinterpret_cast<TinyShared*>(smw)[warp];
    const uint32_t task = ids[slot];
    const STask tk = tasks[task];
    const uint32_t n = tk.count;
    for (uint32_t i = lane; i < n; i += 32) {
        const uint32_t e = perm[tk.start + i];
        w.lo[i] = box[2ull * e];
        w.hi[i] = box[2ull * e + 1];
        w.cen[i] = cen[e];
        w.sidx[i] = e;
        w.ord[i] = (uint16_t)i;
    }
    if (lane == 0) {
        w.fs[0] = 0; w.fc[0] = n; w.fpatch[0] = 0xFFFFFFFFu; w.fdepth[0] = 1;
        w.sp = 1;
        w.node_count = 0;
        w.max_depth = 0;
        w.max_leaf = 0;
        w.bad = 0;
    }
    __syncwarp();
    SrGpuNode* o = out + 2ull * tk.start;
    while (true) {
        if (lane == 0) {
            if (w.sp > 0) {
                --w.sp;
                w.cur_s = w.fs[w.sp]; w.cur_c = w.fc[w.sp]; w.cur_patch = w.fpatch[w.sp]; w.cur_depth = w.fdepth[w.sp];
            } else {
                w.cur_c = 0;
            }
        }
        __syncwarp();
        const uint32_t s = w.cur_s, c = w.cur_c;
        if (c == 0) break;
        const bool small_leaf = c <= 3;
        if (small_leaf) {  // a leaf needs only its box: lane 0 takes the min / max of its few boxes
            if (lane == 0) {
                float lo[4] = {INFINITY, INFINITY, INFINITY, INFINITY}, hi[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
                for (uint32_t i = 0; i < c; ++i) {
                    const uint32_t e = w.ord[s + i];
                    const float4 a = w.lo[e], b = w.hi[e];
                    for (int k = 0; k < 4; ++k) { lo[k] = fminf(lo[k], ax(a, k)); hi[k] = fmaxf(hi[k], ax(b, k)); }
                }
                const int idx = w.node_count++;
                SrGpuNode nd;
                for (int k = 0; k < 4; ++k) { nd.min[k] = lo[k]; nd.max[k] = hi[k]; }
                nd.right_or_first = tk.start + s;
                nd.count = c;
                nd.left = 0;
                nd.pad = 0;
                if ((int)c > w.max_leaf) w.max_leaf = (int)c;
                o[idx] = nd;
                if (w.cur_patch != 0xFFFFFFFFu) o[w.cur_patch].right_or_first = (uint32_t)idx;
                if ((int)w.cur_depth > w.max_depth) w.max_depth = (int)w.cur_depth;
            }
            __syncwarp();
            continue;
        }
        // Bounds and centroid bounds, reduced across the warp.
        float v[16];
        for (int k = 0; k < 4; ++k) { v[k] = INFINITY; v[4 + k] = -INFINITY; v[8 + k] = INFINITY; v[12 + k] = -INFINITY; }
        for (uint32_t i = lane; i < c; i += 32) {
            const uint32_t e = w.ord[s + i];
            const float4 a = w.lo[e], b = w.hi[e], m = w.cen[e];
            for (int k = 0; k < 4; ++k) {
                v[k] = fminf(v[k], ax(a, k));
                v[4 + k] = fmaxf(v[4 + k], ax(b, k));
                v[8 + k] = fminf(v[8 + k], ax(m, k));
                v[12 + k] = fmaxf(v[12 + k], ax(m, k));
            }
        }
        for (int k = 0; k < 16; ++k) {
            const bool mx = (k / 4) % 2 == 1;
            float x = v[k];
            for (int off = 16; off > 0; off >>= 1) {
                const float y = __shfl_xor_sync(0xFFFFFFFFu, x, off);
                x = mx ? fmaxf(x, y) : fminf(x, y);
            }
            v[k] = x;
        }
        if (lane == 0)
            for (int k = 0; k < 16; ++k) w.red[k] = okey(v[k]);
        for (uint32_t j = lane; j < 128; j += 32) { (&w.bl[0][0])[j] = okey(INFINITY); (&w.bh[0][0])[j] = okey(-INFINITY); }
        w.bc[lane] = 0;
        __syncwarp();
        {
            float amin[4], inv[4];
            bool live[4];
            for (int a = 0; a < 4; ++a) {
                amin[a] = oval(w.red[8 + a]);
                const float ext = oval(w.red[12 + a]) - amin[a];
                inv[a] = 8.0f / ext;
                live[a] = ext >= 1e-4f;
            }
            for (uint32_t i = lane; i < c; i += 32) {
                const uint32_t e = w.ord[s + i];
                const float4 a = w.lo[e], b = w.hi[e], m = w.cen[e];
                for (int x = 0; x < 4; ++x) {
                    if (!live[x]) continue;
                    const int bi = x * BINS + bin_of(ax(m, x), amin[x], inv[x]);
                    for (int k = 0; k < 4; ++k) {
                        atomicMin(&w.bl[bi][k], okey(ax(a, k)));
                        atomicMax(&w.bh[bi][k], okey(ax(b, k)));
                    }
                    atomicAdd(&w.bc[bi], 1u);
                }
            }
            __syncwarp();
        }
        const SplitChoice ch = decide_split_warp(w.red + 8, w.red + 12, w.bl, w.bh, w.bc, lane);
        if (lane == 0) {
            int leaf = ch.leaf, axis = ch.axis;
            const float pos = ch.pos;
            uint32_t mid = 0;
            if (!leaf) {
                // The reference's partition pass.
                for (uint32_t i = 0; i < c; ++i) {
                    const uint16_t e = w.ord[s + i];
                    if (ax(w.cen[e], axis) < pos) {
                        w.ord[s + i] = w.ord[s + mid];
                        w.ord[s + mid] = e;
                        ++mid;
                    }
                }
                if (mid == 0 || mid == c) {  // the reference selects by median here: not supported
                    w.bad = 1;
                    leaf = 1;
                }
            }
            const int idx = w.node_count++;
            SrGpuNode nd;
            for (int k = 0; k < 4; ++k) { nd.min[k] = oval(w.red[k]); nd.max[k] = oval(w.red[4 + k]); }
            if (leaf) {
                nd.right_or_first = tk.start + s;
                nd.count = c;
                nd.left = 0;
                if ((int)c > w.max_leaf) w.max_leaf = (int)c;
            } else {
                nd.right_or_first = 0;
                nd.count = 0;
                nd.left = (uint32_t)idx + 1;
            }
            nd.pad = 0;
            o[idx] = nd;
            if (w.cur_patch != 0xFFFFFFFFu) o[w.cur_patch].right_or_first = (uint32_t)idx;
            if ((int)w.cur_depth > w.max_depth) w.max_depth = (int)w.cur_depth;
            if (!leaf) {
                if (w.sp + 2 > 64) {
                    w.bad = 2;
                } else {
                    w.fs[w.sp] = s + mid; w.fc[w.sp] = c - mid; w.fpatch[w.sp] = (uint32_t)idx; w.fdepth[w.sp] = w.cur_depth + 1; ++w.sp;
                    w.fs[w.sp] = s; w.fc[w.sp] = mid; w.fpatch[w.sp] = 0xFFFFFFFFu; w.fdepth[w.sp] = w.cur_depth + 1; ++w.sp;
                }
            }
        }
        __syncwarp();
    }
    for (uint32_t i = lane; i < n; i += 32) perm[tk.start + i] = w.sidx[w.ord[i]];
    if (lane == 0) res[task] = SResult{(uint32_t)w.node_count, (uint32_t)w.max_depth, (uint32_t)w.max_leaf, (uint32_t)w.bad};
}

// Small subtree nodes into the final array at `base` (links made absolute).
__global__ void k_place_small(const STask* tasks, const SResult* res, const uint32_t* base, const SrGpuNode* tmp,
                              SrGpuNode* nodes) {
    const STask tk = tasks[blockIdx.x];
    const uint32_t b = base[blockIdx.x], cnt = res[blockIdx.x].nodes;
    for (uint32_t j = threadIdx.x; j < cnt; j += blockDim.x) {
        SrGpuNode nd = tmp[2ull * tk.start + j];
        if (nd.count == 0) {
            nd.left += b;
            nd.right_or_first += b;
        }
        nodes[b + j] = nd;
    }
}

__global__ void k_place_large(const SrGpuNode* src, const uint32_t* at, uint32_t cnt, SrGpuNode* nodes) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < cnt) nodes[at[j]] = src[j];
}

// Build scratch from the stream-ordered pool (freed in stream order when the buffer goes out of
// scope), so that small scenes rebuilt every frame do not pay cudaMalloc / cudaFree each time.
template <class T>
struct Buf {
    T* p = nullptr;
    cudaStream_t st = nullptr;
    ~Buf() { if (p) cudaFreeAsync(p, st); }
    cudaError_t alloc(size_t n, cudaStream_t s) {
        st = s;
        return cudaMallocAsync(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T), s);
    }
};

}  // namespace

// Keeps the device's stream-ordered pool from returning memory at every synchronisation (once
// per device), so that repeated builds reuse it.
cudaError_t keep_build_pool() {
    static std::mutex mu;
    static std::vector<int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return cudaSuccess;
    cudaMemPool_t pool;
    if ((e = cudaDeviceGetDefaultMemPool(&pool, dev)) != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    done.push_back(dev);
    return cudaSuccess;
}

// Hot (5 float4) and cold (12 float4) records from build order into leaf order.
__global__ void k_gather_records(const uint32_t* order, uint32_t n, const float4* gin, const float4* ain, float4* gout,
                                 float4* aout) {
    const uint64_t total = 17ull * n;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < total; j += (uint64_t)gridDim.x * blockDim.x) {
        if (j < 5ull * n) {
            const uint64_t r = j / 5, k = j % 5;
            gout[j] = gin[5ull * order[r] + k];
        } else {
            const uint64_t jj = j - 5ull * n, r = jj / 12, k = jj % 12;
            aout[jj] = ain[12ull * order[r] + k];
        }
    }
}

cudaError_t gpu_gather_records(const uint32_t* order, uint32_t n, const SrGpuGeom* gin, const SrGpuAttr* ain,
                               SrGpuGeom* gout, SrGpuAttr* aout, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_gather_records<<<148 * 16, 256, 0, st>>>(order, n, reinterpret_cast<const float4*>(gin),
                                                reinterpret_cast<const float4*>(ain), reinterpret_cast<float4*>(gout),
                                                reinterpret_cast<float4*>(aout));
    return cudaGetLastError();
}

cudaError_t gpu_bvh_build_forest(const float4* box, uint32_t n, const GpuSegment* seg, uint32_t num_seg,
                                 SrGpuNode* nodes, uint32_t* order, GpuTreeInfo* tree, GpuBuildInfo* info,
                                 cudaStream_t st) {
    *info = GpuBuildInfo{};
    for (uint32_t s = 0; s < num_seg; ++s) tree[s] = GpuTreeInfo{0, 0, 0, 0};
    if (n == 0) return cudaSuccess;
    cudaError_t e = keep_build_pool();
    if (e != cudaSuccess) return e;
#define BK(x) do { if ((e = (x)) != cudaSuccess) return e; } while (0)
    Buf<float4> cen;
    Buf<uint32_t> perm, perm2, flag, key, lb, svc, sb;
    Buf<int> ei[2], er[2];
    Buf<SrGpuNode> tmp;
    BK(cen.alloc(n, st));
    BK(perm.alloc(n, st));
    BK(perm2.alloc(n, st));
    BK(tmp.alloc(2ull * n, st));
    k_init_build<<<(n + 255) / 256, 256, 0, st>>>(box, n, cen.p, perm.p);
    BK(cudaGetLastError());

    // Host view of the large nodes: bounds, children and the small subtree at each leaf of this
    // part of the tree; `seg` is the tree the node belongs to.
    struct HNode {
        float lo[4], hi[4];
        uint32_t start, count, seg;
        int left = -1, right = -1, small = -1, leaf = 0;
    };
    std::vector<HNode> hn;
    std::vector<STask> small;
    std::vector<int> small_owner;
    std::vector<uint32_t> level;  // hn ids of this level's large nodes
    std::vector<int> root(num_seg, -1);
    bool any_large = false;
    for (uint32_t sg = 0; sg < num_seg; ++sg) {
        if (seg[sg].count == 0) continue;
        HNode r{};
        r.start = seg[sg].start;
        r.count = seg[sg].count;
        r.seg = sg;
        root[sg] = (int)hn.size();
        if (r.count > SMALL) {
            level.push_back((uint32_t)hn.size());
            any_large = true;
        } else {
            r.small = (int)small.size();
            small.push_back({r.start, r.count});
            small_owner.push_back((int)hn.size());
        }
        hn.push_back(r);
    }
    size_t scan_bytes = 0;
    Buf<unsigned char> scan_tmp;
    if (any_large) {
        cub::DeviceScan::ExclusiveSumByKey(nullptr, scan_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                           (uint32_t*)nullptr, (int)n);
        BK(scan_tmp.alloc(scan_bytes, st));
        BK(flag.alloc(n, st));
        BK(key.alloc(n, st));
        BK(lb.alloc(n, st));
        BK(svc.alloc(n, st));
        BK(sb.alloc(n, st));
        for (int k = 0; k < 2; ++k) { BK(ei[k].alloc(2ull * n, st)); BK(er[k].alloc(2ull * n, st)); }
    }
    while (!level.empty()) {
        const uint32_t nt = (uint32_t)level.size();
        std::vector<LTask> tasks(nt);
        std::vector<Chunk> chunks;
        uint32_t q = 0;
        for (uint32_t t = 0; t < nt; ++t) {
            const HNode& h = hn[level[t]];
            tasks[t] = {h.start, h.count, q};
            for (uint32_t c0 = 0; c0 < h.count; c0 += CHUNK) chunks.push_back({t, q + c0, q + std::min(h.count, c0 + CHUNK)});
            q += h.count;
        }
        const uint32_t total = q, nch = (uint32_t)chunks.size();
        Buf<LTask> dt;
        Buf<Chunk> dc;
        Buf<LHead> dh;
        Buf<LBins> db;
        BK(dt.alloc(nt, st));
        BK(dc.alloc(nch, st));
        BK(dh.alloc(nt, st));
        BK(db.alloc(nt, st));
        BK(cudaMemcpyAsync(dt.p, tasks.data(), nt * sizeof(LTask), cudaMemcpyHostToDevice, st));
        BK(cudaMemcpyAsync(dc.p, chunks.data(), nch * sizeof(Chunk), cudaMemcpyHostToDevice, st));
        k_init_heads<<<nt, 128, 0, st>>>(dh.p, db.p, nt);
        k_large_bounds<<<nch, 256, 0, st>>>(dc.p, dt.p, perm.p, box, cen.p, dh.p);
        k_large_bins<<<nch, 256, 0, st>>>(dc.p, dt.p, perm.p, box, cen.p, dh.p, db.p);
        k_large_decide<<<(nt + 127) / 128, 128, 0, st>>>(dh.p, db.p, nt);
        k_large_flags<<<nch, 256, 0, st>>>(dc.p, dt.p, dh.p, perm.p, cen.p, flag.p, key.p);
        BK(cudaGetLastError());
        BK(cub::DeviceScan::ExclusiveSumByKey(scan_tmp.p, scan_bytes, key.p, flag.p, lb.p, (int)total, cub::Equality(), st));
        k_large_service<<<nch, 256, 0, st>>>(dc.p, dt.p, flag.p, lb.p, svc.p);
        BK(cub::DeviceScan::ExclusiveSumByKey(scan_tmp.p, scan_bytes, key.p, svc.p, sb.p, (int)total, cub::Equality(), st));
        BK(cudaMemsetAsync(ei[0].p, 0xFF, 2ull * total * sizeof(int), st));
        BK(cudaMemsetAsync(er[0].p, 0xFF, 2ull * total * sizeof(int), st));
        k_large_events<<<nch, 256, 0, st>>>(dc.p, dt.p, perm.p, flag.p, lb.p, svc.p, sb.p, ei[0].p, er[0].p, dh.p);
        BK(cudaGetLastError());
        // A chain of references in a node's enqueue list is shorter than the list (at most twice
        // the node's size), and every round halves it: log2 of that many rounds resolve all.
        int cur = 0;
        const uint32_t len = 2u * total;
        uint32_t maxc = 0;
        for (const LTask& tk : tasks) maxc = std::max(maxc, tk.count);
        int rounds = 1;
        while ((1ull << rounds) < 2ull * maxc + 2) ++rounds;
        for (int round = 0; round <= rounds; ++round) {
            k_jump<<<(len + 255) / 256, 256, 0, st>>>(ei[cur].p, er[cur].p, ei[1 - cur].p, er[1 - cur].p, len);
            BK(cudaGetLastError());
            cur = 1 - cur;
        }
        k_large_scatter<<<nch, 256, 0, st>>>(dc.p, dt.p, dh.p, perm.p, flag.p, lb.p, ei[cur].p, perm2.p);
        k_copy_range<<<nch, 256, 0, st>>>(dc.p, dt.p, perm2.p, perm.p);
        BK(cudaGetLastError());
        std::vector<LHead> heads(nt);
        BK(cudaMemcpyAsync(heads.data(), dh.p, nt * sizeof(LHead), cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
        std::vector<uint32_t> next;
        for (uint32_t t = 0; t < nt; ++t) {
            const LHead& h = heads[t];
            const uint32_t id = level[t];
            for (int k = 0; k < 4; ++k) { hn[id].lo[k] = oval_host(h.blo[k]); hn[id].hi[k] = oval_host(h.bhi[k]); }
            if (h.leaf) {
                hn[id].leaf = 1;
                GpuTreeInfo& ti = tree[hn[id].seg];
                ti.max_leaf = std::max(ti.max_leaf, hn[id].count);
                continue;
            }
            if (h.m == 0 || h.m == hn[id].count) {
                info->unsupported = 1;
                return cudaSuccess;
            }
            const uint32_t s = hn[id].start, c = hn[id].count;
            const uint32_t parts[2][2] = {{s, h.m}, {s + h.m, c - h.m}};
            for (int side = 0; side < 2; ++side) {
                HNode ch{};
                ch.start = parts[side][0];
                ch.count = parts[side][1];
                ch.seg = hn[id].seg;
                const int cid = (int)hn.size();
                if (ch.count > SMALL) {
                    next.push_back((uint32_t)cid);
                } else {
                    ch.small = (int)small.size();
                    small.push_back({ch.start, ch.count});
                    small_owner.push_back(cid);
                }
                hn.push_back(ch);
                if (side == 0) hn[id].left = cid;
                else hn[id].right = cid;
            }
        }
        level.swap(next);
    }

    // Small subtrees.
    const uint32_t ns = (uint32_t)small.size();
    Buf<STask> dst;
    Buf<SResult> dres;
    std::vector<SResult> res(ns);
    if (ns) {
        BK(dst.alloc(ns, st));
        BK(dres.alloc(ns, st));
        BK(cudaMemcpyAsync(dst.p, small.data(), ns * sizeof(STask), cudaMemcpyHostToDevice, st));
        // Subtrees of at most TINY primitives one warp each, the others one block each.
        std::vector<uint32_t> ids;
        uint32_t n_tiny = 0;
        for (uint32_t k = 0; k < ns; ++k)
            if (small[k].count <= TINY) ids.push_back(k);
        n_tiny = (uint32_t)ids.size();
        for (uint32_t k = 0; k < ns; ++k)
            if (small[k].count > TINY) ids.push_back(k);
        Buf<uint32_t> dids;
        BK(dids.alloc(ns, st));
        BK(cudaMemcpyAsync(dids.p, ids.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        if (n_tiny) {
            const size_t smem_w = WARPS_TINY * sizeof(TinyShared);
            BK(cudaFuncSetAttribute(k_small_build_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_w));
            k_small_build_warp<<<(n_tiny + WARPS_TINY - 1) / WARPS_TINY, 32 * WARPS_TINY, smem_w, st>>>(
                dst.p, dids.p, n_tiny, box, cen.p, perm.p, tmp.p, dres.p);
        }
        if (ns > n_tiny) {
            const size_t smem = 3 * SMALL * sizeof(float4) + SMALL * (sizeof(uint32_t) + sizeof(uint16_t));
            BK(cudaFuncSetAttribute(k_small_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_small_build<<<ns - n_tiny, 256, smem, st>>>(dst.p, dids.p + n_tiny, box, cen.p, perm.p, tmp.p, dres.p);
        }
        BK(cudaGetLastError());
        BK(cudaMemcpyAsync(res.data(), dres.p, ns * sizeof(SResult), cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
    }
    for (uint32_t k = 0; k < ns; ++k) {
        if (res[k].bad) { info->unsupported = 1; return cudaSuccess; }
        GpuTreeInfo& ti = tree[hn[small_owner[k]].seg];
        ti.max_leaf = std::max(ti.max_leaf, res[k].max_leaf);
    }

    // Depth-first numbering of the large nodes and the small subtrees' bases, tree after tree.
    std::vector<uint32_t> pre(hn.size(), 0), sbase(ns, 0);
    std::vector<SrGpuNode> lnodes;
    std::vector<uint32_t> lat;
    uint32_t nextidx = 0;
    struct Fr { int id; uint32_t d; };
    std::vector<Fr> stack;
    for (uint32_t sg = 0; sg < num_seg; ++sg) {
        GpuTreeInfo& ti = tree[sg];
        ti.node_base = nextidx;
        if (root[sg] < 0) continue;
        uint32_t depth = 0;
        stack.push_back({root[sg], 1});
        while (!stack.empty()) {
            Fr f = stack.back();
            stack.pop_back();
            HNode& h = hn[f.id];
            pre[f.id] = nextidx;
            if (h.small >= 0) {
                sbase[h.small] = nextidx;
                nextidx += res[h.small].nodes;
                depth = std::max(depth, f.d - 1 + res[h.small].depth);
                continue;
            }
            depth = std::max(depth, f.d);
            ++nextidx;
            if (!h.leaf) {
                stack.push_back({h.right, f.d + 1});
                stack.push_back({h.left, f.d + 1});
            }
        }
        ti.num_nodes = nextidx - ti.node_base;
        ti.depth = depth;
        info->depth = std::max(info->depth, depth);
        info->max_leaf = std::max(info->max_leaf, ti.max_leaf);
    }
    for (size_t id = 0; id < hn.size(); ++id) {
        const HNode& h = hn[id];
        if (h.small >= 0) continue;
        SrGpuNode nd;
        for (int k = 0; k < 4; ++k) { nd.min[k] = h.lo[k]; nd.max[k] = h.hi[k]; }
        if (h.leaf) {
            nd.right_or_first = h.start;
            nd.count = h.count;
            nd.left = 0;
        } else {
            nd.right_or_first = pre[h.right];
            nd.count = 0;
            nd.left = pre[h.left];
        }
        nd.pad = 0;
        lnodes.push_back(nd);
        lat.push_back(pre[id]);
    }
    Buf<SrGpuNode> dl;
    Buf<uint32_t> dlat, dsb;
    BK(dl.alloc(lnodes.size(), st));
    BK(dlat.alloc(lat.size(), st));
    BK(dsb.alloc(ns, st));
    BK(cudaMemcpyAsync(dl.p, lnodes.data(), lnodes.size() * sizeof(SrGpuNode), cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(dlat.p, lat.data(), lat.size() * 4, cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(dsb.p, sbase.data(), ns * 4, cudaMemcpyHostToDevice, st));
    if (!lnodes.empty())
        k_place_large<<<((uint32_t)lnodes.size() + 255) / 256, 256, 0, st>>>(dl.p, dlat.p, (uint32_t)lnodes.size(), nodes);
    if (ns) k_place_small<<<ns, 256, 0, st>>>(dst.p, dres.p, dsb.p, tmp.p, nodes);
    BK(cudaGetLastError());
    BK(cudaMemcpyAsync(order, perm.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
    BK(cudaStreamSynchronize(st));
    info->num_nodes = nextidx;
#undef BK
    return cudaSuccess;
}

cudaError_t gpu_bvh_build(const float4* box, uint32_t n, SrGpuNode* nodes, uint32_t* order, GpuBuildInfo* info,
                          cudaStream_t st) {
    const GpuSegment all{0, n};
    GpuTreeInfo tree{};
    return gpu_bvh_build_forest(box, n, &all, 1, nodes, order, &tree, info, st);
}

}  // namespace srk
