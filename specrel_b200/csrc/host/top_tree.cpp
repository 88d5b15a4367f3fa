// top_tree (bvh4d.rs:593-644): the tree over an arena's chunks, a full-sweep SAH over their boxes
// with the chunks' simplex counts as weights. The reference sorts its items in place, stably, by
// the box centre on each axis in turn (f32::total_cmp), sweeps each order for the cheapest split,
// sorts once more by the best axis and recurses left then right. This computes the same tree
// (the same sort orders, float operations and tie-breaks) faster: items are sorted as indices on
// precomputed integer keys, and each node's order on every axis is handed down to its children by
// a stable partition. A child whose inherited order has no ties on an axis takes it as is (a strict
// order is what any stable sort gives); only orders with ties are sorted again, by an
// allocation-free stable merge sort, from the order the reference sorts. A subtree over m items
// has m - 1 nodes, so each subtree's node slots are known before it is built, and subtrees of 256
// items or more are built on threads of their own.
#include <immintrin.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <vector>

#include "../../../include/specrel.h"
#include "../../../include/specrel_scene.h"

namespace {

inline int32_t total_key(float f) {  // f32::total_cmp as an integer order
    int32_t b;
    std::memcpy(&b, &f, 4);
    return b ^ (int32_t)((uint32_t)(b >> 31) >> 1);
}

// Aabb4D::union. Boxes hold no NaN and no -0 (simplex boxes are padded by 1e-4), where SSE's
// min / max (and a compare-select) give f32::min / max's values.
struct Box4 {
    __m128 lo, hi;
};
inline Box4 empty4() { return {_mm_set1_ps(INFINITY), _mm_set1_ps(-INFINITY)}; }
inline void unite4(Box4& b, const float* item) {
    b.lo = _mm_min_ps(b.lo, _mm_loadu_ps(item));
    b.hi = _mm_max_ps(b.hi, _mm_loadu_ps(item + 4));
}
inline float measure4(const Box4& b) {  // box_measure (bvh4d.rs:8-13) on (t, x, y, z) lanes
    alignas(16) float e[4];
    _mm_store_ps(e, _mm_sub_ps(b.hi, b.lo));
    const float spatial = e[1] * e[2] + e[2] * e[3] + e[3] * e[1];
    const float temporal = 0.22f * e[0] * (e[1] + e[2] + e[3]);
    return spatial + temporal;
}

struct Builder {
    const float* box;  // item i: box[8i .. 8i+3] = lo, box[8i+4 .. 8i+7] = hi
    const uint32_t* root;
    const float* weight;
    const uint32_t* depth;
    uint32_t base;
    std::vector<int32_t> key[4];    // key[a][i]: total order of item i's centre on axis a
    std::vector<uint32_t> order;    // the items, in the reference's current in-place order
    std::vector<uint32_t> buf;      // merge scratch
    std::vector<uint32_t> saved[4]; // saved[a][lo, hi): the node's items in its order on axis a
    std::vector<uint8_t> side;      // per item: 0 left, 1 right of the current split
    std::vector<float> rm, rw;  // per position: the right side's measure and weight
    std::vector<SrGpuNode> out;

    // Stable sort of v[0, n) by k: insertion-sorted runs of 16, then bottom-up merges through
    // `scratch` (n entries).
    static void stable_sort(uint32_t* v, size_t n, const int32_t* k, uint32_t* scratch) {
        const size_t RUN = 16;
        for (size_t s = 0; s < n; s += RUN) {
            const size_t e = std::min(n, s + RUN);
            for (size_t i = s + 1; i < e; ++i) {
                const uint32_t x = v[i];
                const int32_t kx = k[x];
                size_t j = i;
                while (j > s && k[v[j - 1]] > kx) {
                    v[j] = v[j - 1];
                    --j;
                }
                v[j] = x;
            }
        }
        if (n <= RUN) return;
        uint32_t* src = v;
        uint32_t* dst = scratch;
        for (size_t w = RUN; w < n; w *= 2) {
            for (size_t s = 0; s < n; s += 2 * w) {
                const size_t m = std::min(n, s + w), e = std::min(n, s + 2 * w);
                size_t i = s, j = m, o = s;
                while (i < m && j < e) dst[o++] = (k[src[j]] < k[src[i]]) ? src[j++] : src[i++];
                while (i < m) dst[o++] = src[i++];
                while (j < e) dst[o++] = src[j++];
            }
            std::swap(src, dst);
        }
        if (src != v) std::memcpy(v, src, n * sizeof(uint32_t));
    }

    // Whether the items of v[0, n) are in strictly increasing key order.
    static bool strict(const uint32_t* v, size_t n, const int32_t* k) {
        for (size_t i = 1; i < n; ++i)
            if (!(k[v[i - 1]] < k[v[i]])) return false;
        return true;
    }

    // Stable partition of v[0, n) by side: the left items first.
    void partition(uint32_t* v, size_t n, uint32_t* scratch) {
        size_t l = 0, r = 0;
        for (size_t i = 0; i < n; ++i) {
            if (side[v[i]] == 0) v[l++] = v[i];
            else scratch[r++] = v[i];
        }
        std::memcpy(v + l, scratch, r * sizeof(uint32_t));
    }

    // The subtree over order[a, b); returns its node index and raises `max_d` to its depth.
    // `levels`: tree nodes above it. `inherited`: saved[*][a, b) holds the parent's orders
    // restricted to these items. Its nodes take out[slot, slot + b - a - 1) in depth-first order
    // (a subtree over m items has m - 1 nodes), so subtrees can be built concurrently; every
    // scratch array is used in the subtree's own range [a, b).
    uint32_t build(size_t a, size_t b, uint32_t levels, bool inherited, size_t slot, uint32_t& max_d, int spawn) {
        const size_t n = b - a;
        if (n == 1) {
            const uint32_t it = order[a];
            max_d = std::max(max_d, levels + depth[it]);
            return root[it];
        }
        const uint32_t at = slot == 0 ? 0u : base + (uint32_t)slot - 1;
        uint32_t* scratch = buf.data() + a;
        float* rm_ = rm.data() + a;
        float* rw_ = rw.data() + a;
        Box4 bounds = empty4();
        for (size_t i = a; i < b; ++i) unite4(bounds, box + 8 * order[i]);

        float best_cost = INFINITY;
        int best_axis = 0;
        size_t best_mid = n / 2;
        uint32_t* v = order.data() + a;
        for (int axis = 0; axis < 4; ++axis) {
            // The reference's stable sort of the current order by this axis.
            uint32_t* sv = saved[axis].data() + a;
            if (inherited && strict(sv, n, key[axis].data())) {
                std::memcpy(v, sv, n * sizeof(uint32_t));
            } else {
                stable_sort(v, n, key[axis].data(), scratch);
                std::memcpy(sv, v, n * sizeof(uint32_t));
            }
            // The right sides' boxes accumulated from the end (their measures kept), then the
            // left sides' from the front: cost = left weight * measure + right weight * measure.
            Box4 acc = empty4();
            float aw = 0.0f;
            for (size_t j = n - 1; j >= 1; --j) {
                const uint32_t it = v[j];
                unite4(acc, box + 8 * it);
                aw = aw + weight[it];
                rm_[j] = measure4(acc);
                rw_[j] = aw;
            }
            Box4 left_box = empty4();
            float lw = 0.0f;
            for (size_t j = 1; j < n; ++j) {
                const uint32_t it = v[j - 1];
                unite4(left_box, box + 8 * it);
                lw = lw + weight[it];
                const float cost = lw * measure4(left_box) + rw_[j] * rm_[j];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_mid = j;
                }
            }
        }
        if (best_axis != 3) {
            // The reference sorts the axis-3 order by the best axis. Without ties on that axis the
            // result is the one strict order, which the best axis's own sort already gave.
            const int32_t* k = key[best_axis].data();
            const uint32_t* sv = saved[best_axis].data() + a;
            if (strict(sv, n, k)) std::memcpy(v, sv, n * sizeof(uint32_t));
            else stable_sort(v, n, k, scratch);
        }
        for (size_t i = 0; i < n; ++i) side[v[i]] = i < best_mid ? 0 : 1;
        for (int axis = 0; axis < 4; ++axis) partition(saved[axis].data() + a, n, scratch);
        // Left subtree's nodes from slot + 1 (best_mid - 1 of them), the right's after them.
        uint32_t left, right;
        if (spawn > 0 && best_mid >= PAR_MIN && n - best_mid >= PAR_MIN) {
            uint32_t dl = 0;
            auto fut = std::async(std::launch::async, [&] {
                return build(a, a + best_mid, levels + 1, true, slot + 1, dl, spawn - 1);
            });
            right = build(a + best_mid, b, levels + 1, true, slot + best_mid, max_d, spawn - 1);
            left = fut.get();
            max_d = std::max(max_d, dl);
        } else {
            left = build(a, a + best_mid, levels + 1, true, slot + 1, max_d, 0);
            right = build(a + best_mid, b, levels + 1, true, slot + best_mid, max_d, 0);
        }
        SrGpuNode nd{};
        _mm_storeu_ps(nd.min, bounds.lo);
        _mm_storeu_ps(nd.max, bounds.hi);
        nd.right_or_first = right;
        nd.count = 0;
        nd.left = left;
        out[slot] = nd;
        return at;
    }
    static constexpr size_t PAR_MIN = 256;  // items of a subtree worth a thread of its own
};

}  // namespace

extern "C" sr_status sr_top_tree(const float* boxes, const uint32_t* roots, const float* weights,
                                 const uint32_t* depths, uint32_t n, uint32_t base, SrGpuNode* nodes,
                                 uint32_t* depth) {
    if (n < 2 || !boxes || !roots || !weights || !nodes) return SR_ERR_INVALID_ARGUMENT;
    Builder bld;
    bld.box = boxes;
    bld.root = roots;
    bld.weight = weights;
    std::vector<uint32_t> zero;
    if (!depths) zero.assign(n, 0);
    bld.depth = depths ? depths : zero.data();
    bld.base = base;
    for (int a = 0; a < 4; ++a) {
        bld.key[a].resize(n);
        for (uint32_t i = 0; i < n; ++i) bld.key[a][i] = total_key((boxes[8 * i + a] + boxes[8 * i + 4 + a]) * 0.5f);
        bld.saved[a].resize(n);
    }
    bld.side.resize(n);
    bld.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) bld.order[i] = i;
    bld.buf.resize(n);
    bld.rm.resize(n);
    bld.rw.resize(n);
    bld.out.resize(n - 1);
    uint32_t max_d = 0;
    bld.build(0, n, 0, false, 0, max_d, 2);
    std::memcpy(nodes, bld.out.data(), bld.out.size() * sizeof(SrGpuNode));
    if (depth) *depth = max_d;
    return SR_OK;
}
