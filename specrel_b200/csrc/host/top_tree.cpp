// top_tree (bvh4d.rs:593-644): the tree over an arena's chunks, a full-sweep SAH over their boxes
// with the chunks' simplex counts as weights. The reference sorts its items in place, stably, by
// the box centre on each axis in turn (f32::total_cmp), sweeps each order for the cheapest split,
// sorts once more by the best axis and recurses left then right. This computes the same tree
// (the same sort orders, float operations and tie-breaks) faster: items are sorted as indices on
// precomputed integer keys, and each node's order on every axis is handed down to its children by
// a stable partition. A child whose inherited order has no ties on an axis takes it as is (a strict
// order is what any stable sort gives); only orders with ties are sorted again, by an
// allocation-free stable merge sort, from the order the reference sorts.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../../include/specrel.h"
#include "../../../include/specrel_scene.h"

namespace {

inline int32_t total_key(float f) {  // f32::total_cmp as an integer order
    int32_t b;
    std::memcpy(&b, &f, 4);
    return b ^ (int32_t)((uint32_t)(b >> 31) >> 1);
}

inline float box_measure(const float* lo, const float* hi) {  // bvh4d.rs:8-13, (t, x, y, z)
    const float et = hi[0] - lo[0], ex = hi[1] - lo[1], ey = hi[2] - lo[2], ez = hi[3] - lo[3];
    const float spatial = ex * ey + ey * ez + ez * ex;
    const float temporal = 0.22f * et * (ex + ey + ez);
    return spatial + temporal;
}

// Aabb4D::union. Boxes hold no NaN and no -0 (simplex boxes are padded by 1e-4), where a
// compare-select gives f32::min / max's values without a libm call.
inline void unite(float* lo, float* hi, const float* blo, const float* bhi) {
    for (int k = 0; k < 4; ++k) {
        lo[k] = blo[k] < lo[k] ? blo[k] : lo[k];
        hi[k] = bhi[k] > hi[k] ? bhi[k] : hi[k];
    }
}

inline void empty_box(float* lo, float* hi) {
    for (int k = 0; k < 4; ++k) {
        lo[k] = INFINITY;
        hi[k] = -INFINITY;
    }
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
    std::vector<float> rlo, rhi, rw;
    std::vector<SrGpuNode> out;
    uint32_t max_depth = 0;

    // Stable sort of v[0, n) by k: insertion-sorted runs of 16, then bottom-up merges.
    void stable_sort(uint32_t* v, size_t n, const int32_t* k) {
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
        uint32_t* dst = buf.data();
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
    void partition(uint32_t* v, size_t n) {
        size_t l = 0, r = 0;
        for (size_t i = 0; i < n; ++i) {
            if (side[v[i]] == 0) v[l++] = v[i];
            else buf[r++] = v[i];
        }
        std::memcpy(v + l, buf.data(), r * sizeof(uint32_t));
    }

    // The subtree over order[a, b); returns its node index. `levels`: tree nodes above it.
    // `inherited`: saved[*][a, b) holds the parent's orders restricted to these items.
    uint32_t build(size_t a, size_t b, uint32_t levels, bool inherited) {
        const size_t n = b - a;
        if (n == 1) {
            const uint32_t it = order[a];
            max_depth = std::max(max_depth, levels + depth[it]);
            return root[it];
        }
        const size_t slot = out.size();
        SrGpuNode blank{};
        out.push_back(blank);
        const uint32_t at = slot == 0 ? 0u : base + (uint32_t)slot - 1;
        float blo[4], bhi[4];
        empty_box(blo, bhi);
        for (size_t i = a; i < b; ++i) unite(blo, bhi, box + 8 * order[i], box + 8 * order[i] + 4);

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
                stable_sort(v, n, key[axis].data());
                std::memcpy(sv, v, n * sizeof(uint32_t));
            }
            float alo[4], ahi[4];
            empty_box(alo, ahi);
            float aw = 0.0f;
            for (size_t j = n - 1; j >= 1; --j) {
                const uint32_t it = v[j];
                unite(alo, ahi, box + 8 * it, box + 8 * it + 4);
                aw = aw + weight[it];
                std::memcpy(&rlo[4 * j], alo, 16);
                std::memcpy(&rhi[4 * j], ahi, 16);
                rw[j] = aw;
            }
            float llo[4], lhi[4];
            empty_box(llo, lhi);
            float lw = 0.0f;
            for (size_t j = 1; j < n; ++j) {
                const uint32_t it = v[j - 1];
                unite(llo, lhi, box + 8 * it, box + 8 * it + 4);
                lw = lw + weight[it];
                const float cost = lw * box_measure(llo, lhi) + rw[j] * box_measure(&rlo[4 * j], &rhi[4 * j]);
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
            else stable_sort(v, n, k);
        }
        for (size_t i = 0; i < n; ++i) side[v[i]] = i < best_mid ? 0 : 1;
        for (int axis = 0; axis < 4; ++axis) partition(saved[axis].data() + a, n);
        const uint32_t left = build(a, a + best_mid, levels + 1, true);
        const uint32_t right = build(a + best_mid, b, levels + 1, true);
        SrGpuNode nd{};
        std::memcpy(nd.min, blo, 16);
        std::memcpy(nd.max, bhi, 16);
        nd.right_or_first = right;
        nd.count = 0;
        nd.left = left;
        out[slot] = nd;
        return at;
    }
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
    bld.rlo.resize(4 * (size_t)n);
    bld.rhi.resize(4 * (size_t)n);
    bld.rw.resize(n);
    bld.out.reserve(n - 1);
    bld.build(0, n, 0, false);
    std::memcpy(nodes, bld.out.data(), bld.out.size() * sizeof(SrGpuNode));
    if (depth) *depth = bld.max_depth;
    return SR_OK;
}
