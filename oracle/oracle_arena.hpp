// TEST INFRASTRUCTURE ONLY — the CPU oracle's restatement of the reference's incremental scene
// cache, used by the parity tests to check the engine's device arena. Restated from:
//   src/dynamic/scene_cache.rs:72-115   Space (first-fit free ranges)
//   src/dynamic/scene_cache.rs:120-356  SceneCache: begin, reuse, install, tube, piece, finish, compact
//   src/dynamic/scene_cache.rs:358-366  push_sample (a chunk's key)
//   src/bvh4d.rs:31-44                  BvhNode4D::NOTHING, moved
//   src/bvh4d.rs:48-61, 157-215, 583-591 BvhVersion, dirty, reset_arena, begin_edit, write_part,
//                                       write_nodes, put
//   src/bvh4d.rs:593-644                top_tree
// The mesh's bits stand for mesh_fingerprint's 64-bit hash of them in a chunk's key (equal keys
// either way, barring a hash collision).
#pragma once
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "oracle_geom.hpp"
#include "oracle_scenes.hpp"

namespace orc {

struct Span {
    size_t lo = 0, hi = 0;
    size_t size() const { return hi - lo; }
    bool none() const { return hi <= lo; }
};

// scene_cache.rs:72-115.
struct FreeList {
    std::vector<Span> free;
    size_t end = 0;
    size_t take(size_t n) {
        auto it = std::find_if(free.begin(), free.end(), [&](const Span& f) { return f.size() >= n; });
        if (it != free.end()) {
            size_t at = it->lo;
            it->lo += n;
            if (it->none()) free.erase(it);
            return at;
        }
        end += n;
        return end - n;
    }
    void give(Span r) {
        if (r.none()) return;
        size_t k = 0;
        while (k < free.size() && free[k].lo < r.lo) ++k;
        free.insert(free.begin() + k, r);
        if (k + 1 < free.size() && free[k].hi == free[k + 1].lo) {
            free[k].hi = free[k + 1].hi;
            free.erase(free.begin() + k + 1);
        }
        if (k > 0 && free[k - 1].hi == free[k].lo) {
            free[k - 1].hi = free[k].hi;
            free.erase(free.begin() + k);
        }
        if (!free.empty() && free.back().hi == end) {
            end = free.back().lo;
            free.pop_back();
        }
    }
    size_t holes() const {
        size_t h = 0;
        for (auto& f : free) h += f.size();
        return h;
    }
};

inline uint64_t next_layout() {
    static uint64_t n = 0;
    return ++n;
}

template <class T> BvhNode<T> nothing() { return BvhNode<T>{}; }  // empty box, no links (bvh4d.rs:31)

// A Bvh used as an arena (bvh4d.rs:168-215, 583-591). Its order is the identity and its simplices
// are kept in leaf order.
template <class T> struct ArenaBvh {
    Bvh<T> b;
    uint64_t layout = 0, edit = 0;             // BvhVersion (bvh4d.rs:48-61)
    std::vector<Span> dirty_nodes, dirty_prims;  // what the latest edit wrote

    void begin_edit() {
        ++edit;
        dirty_nodes.clear();
        dirty_prims.clear();
    }

    template <class V, class F> static void put(std::vector<V>& v, size_t at, size_t n, F item) {
        for (size_t i = 0; i < n; ++i) {
            if (at + i < v.size()) v[at + i] = item(i);
            else v.push_back(item(i));
        }
    }
    void reset() {
        b.nodes.assign(1, nothing<T>());
        b.hot.clear();
        b.order.clear();
        b.simplices.clear();
        layout = next_layout();
        edit = 0;
        dirty_nodes.clear();
        dirty_prims.clear();
    }
    void write_part(const Bvh<T>& src, Span nodes, Span prims, size_t node_at, size_t prim_at) {
        const uint32_t dn = (uint32_t)node_at - (uint32_t)nodes.lo, dp = (uint32_t)prim_at - (uint32_t)prims.lo;
        put(b.nodes, node_at, nodes.size(), [&](size_t i) {
            BvhNode<T> nd = src.nodes[nodes.lo + i];  // BvhNode4D::moved
            if (nd.count > 0) {
                nd.right_or_first += dp;
            } else {
                nd.left += dn;
                nd.right_or_first += dn;
            }
            return nd;
        });
        put(b.hot, prim_at, prims.size(), [&](size_t i) { return src.hot[prims.lo + i]; });
        put(b.order, prim_at, prims.size(), [&](size_t i) { return (uint32_t)(prim_at + i); });
        put(b.simplices, prim_at, prims.size(), [&](size_t i) { return src.leaf_simplex(prims.lo + i); });
        dirty_nodes.push_back(Span{node_at, node_at + nodes.size()});
        dirty_prims.push_back(Span{prim_at, prim_at + prims.size()});
    }
    void write_nodes(size_t at, const BvhNode<T>* nodes, size_t n) {
        put(b.nodes, at, n, [&](size_t i) { return nodes[i]; });
        dirty_nodes.push_back(Span{at, at + n});
    }
};

// top_tree (bvh4d.rs:593-644): a full-sweep SAH over the subtrees' boxes.
template <class T> struct TopItem {
    Aabb<T> box;
    uint32_t root;
    T weight;
};
template <class T> uint32_t top_tree_rec(std::vector<TopItem<T>>& all, size_t lo, size_t hi, uint32_t base,
                                         std::vector<BvhNode<T>>& out) {
    if (hi - lo == 1) return all[lo].root;
    const size_t k = out.size();
    out.push_back(nothing<T>());
    const uint32_t at = k == 0 ? 0u : base + (uint32_t)k - 1;
    Aabb<T> bounds;
    for (size_t i = lo; i < hi; ++i) bounds = bounds.unite(all[i].box);
    const size_t n = hi - lo;
    T best_cost = std::numeric_limits<T>::infinity();
    int best_axis = 0;
    size_t best_mid = n / 2;
    std::vector<Aabb<T>> right_box(n);
    std::vector<T> right_w(n, T(0));
    auto key = [](T v) {  // total order of floats, as f32::total_cmp
        int32_t b;
        std::memcpy(&b, &v, 4);
        return b ^ (int32_t)((uint32_t)(b >> 31) >> 1);
    };
    auto sort_axis = [&](int axis) {
        std::stable_sort(all.begin() + lo, all.begin() + hi, [&](const TopItem<T>& x, const TopItem<T>& y) {
            return key(x.box.center().axis(axis)) < key(y.box.center().axis(axis));
        });
    };
    for (int axis = 0; axis < 4; ++axis) {
        sort_axis(axis);
        Aabb<T> acc;
        T acc_w = 0;
        for (size_t j = n - 1; j >= 1; --j) {
            acc = acc.unite(all[lo + j].box);
            acc_w = acc_w + all[lo + j].weight;
            right_box[j] = acc;
            right_w[j] = acc_w;
        }
        Aabb<T> left;
        T left_w = 0;
        for (size_t j = 1; j < n; ++j) {
            left = left.unite(all[lo + j - 1].box);
            left_w = left_w + all[lo + j - 1].weight;
            T cost = left_w * box_measure(left) + right_w[j] * box_measure(right_box[j]);
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = axis;
                best_mid = j;
            }
        }
    }
    sort_axis(best_axis);
    uint32_t l = top_tree_rec(all, lo, lo + best_mid, base, out);
    uint32_t r = top_tree_rec(all, lo + best_mid, hi, base, out);
    BvhNode<T> nd;
    nd.aabb = bounds;
    nd.right_or_first = r;
    nd.count = 0;
    nd.left = l;
    out[k] = nd;
    return at;
}

struct CachePart {
    uint32_t kind, player;
    uint64_t id;
};
struct CacheChunkId {
    CachePart part;
    int64_t index;
    bool operator<(const CacheChunkId& o) const {
        return std::tie(part.kind, part.player, part.id, index) < std::tie(o.part.kind, o.part.player, o.part.id, o.index);
    }
};
struct CacheStats {  // scene_cache.rs:59-70
    uint64_t chunks_built = 0, chunks_reused = 0, simplices_built = 0, simplices_reused = 0, arena_simplices = 0;
    uint64_t compacted = 0;
};

// SceneCache (scene_cache.rs:120-356).
template <class T> struct SceneCacheOracle {
    struct Chunk {
        std::vector<uint32_t> key;
        Span nodes, prims;
        Aabb<T> bounds;
        std::unique_ptr<Bvh<T>> fresh;
        uint64_t used = 0;
    };
    std::map<CacheChunkId, Chunk> chunks;
    std::vector<CacheChunkId> order;
    uint64_t generation = 0, layout = 0;
    FreeList nodes, prims;
    Span top, vol_nodes, vol_prims;
    CacheStats stats;

    void begin(ArenaBvh<T>& arena) {
        ++generation;
        order.clear();
        stats = CacheStats{};
        if (arena.layout != layout || layout == 0) {
            arena.reset();
            layout = arena.layout;
            chunks.clear();
            nodes = FreeList{};
            nodes.end = 1;
            prims = FreeList{};
            top = Span{};
            vol_nodes = vol_prims = Span{};
        }
        arena.begin_edit();
    }
    bool reuse(const CacheChunkId& id, const std::vector<uint32_t>& key) {
        Chunk& c = chunks[id];
        bool reused = c.used != 0 && c.key == key;
        if (reused) {
            stats.chunks_reused += 1;
            stats.simplices_reused += c.prims.size();
        } else {
            nodes.give(c.nodes);
            prims.give(c.prims);
            c.nodes = c.prims = Span{};
            c.key = key;
        }
        c.used = generation;
        order.push_back(id);
        return reused;
    }
    void install(const CacheChunkId& id, Bvh<T>&& bvh) {
        stats.chunks_built += 1;
        stats.simplices_built += bvh.simplices.size();
        chunks[id].fresh = std::make_unique<Bvh<T>>(std::move(bvh));
    }
    void piece(const CachePart& part, int64_t index, const std::vector<uint32_t>& key,
               const std::vector<Simplex<T>>& simplices) {
        CacheChunkId id{part, index};
        if (!reuse(id, key)) install(id, Bvh<T>::build(simplices));
    }
    static void push_sample(std::vector<uint32_t>& k, const WorldlineSample<T>& s) {
        auto bits = [&](T v) {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            k.push_back(u);
        };
        bits(s.center.t); bits(s.center.x); bits(s.center.y); bits(s.center.z);
        bits(s.proper_time);
        bits(s.phi.x); bits(s.phi.y); bits(s.phi.z);
        bits(s.proper_accel_local.x); bits(s.proper_accel_local.y); bits(s.proper_accel_local.z);
        for (int e = 0; e < 4; ++e) {
            bits(s.tetrad.e[e].t); bits(s.tetrad.e[e].x); bits(s.tetrad.e[e].y); bits(s.tetrad.e[e].z);
        }
    }
    // scene_cache.rs:203-248; `mesh_bits` stands for the mesh's fingerprint.
    void tube(const CachePart& part, const Mesh3D<T>& mesh, const std::vector<uint32_t>& mesh_bits,
              const std::vector<WorldlineSample<T>>& samples, const T* decided, uint32_t material) {
        if (samples.size() < 2) return;
        auto bucket = [&](size_t i) -> int64_t {
            T f = std::floor(samples[i].center.t / T(1));
            if (f != f) return 0;
            if (f >= T(9.2233720368547758e18)) return INT64_MAX;
            if (f <= T(-9.2233720368547758e18)) return INT64_MIN;
            return (int64_t)f;
        };
        size_t first = 0;
        while (first < samples.size() - 1) {
            int64_t b = bucket(first);
            size_t end = first + 1;
            while (end < samples.size() - 1 && bucket(end) == b) ++end;
            std::vector<uint32_t> key{material, decided ? 1u : 0u};
            key.insert(key.end(), mesh_bits.begin(), mesh_bits.end());
            for (size_t i = first; i <= end; ++i) push_sample(key, samples[i]);
            if (decided)
                for (size_t i = first; i <= end; ++i) {
                    uint32_t u;
                    std::memcpy(&u, &decided[i], 4);
                    key.push_back(u);
                }
            CacheChunkId id{part, b};
            if (!reuse(id, key)) {
                std::vector<WorldlineSample<T>> s(samples.begin() + first, samples.begin() + end + 1);
                std::vector<Simplex<T>> out;
                extend_worldtube_simplices(out, mesh, s, decided ? decided + first : nullptr, material);
                install(id, Bvh<T>::build(std::move(out)));
            }
            first = end;
        }
    }
    void compact(ArenaBvh<T>& arena) {  // scene_cache.rs:338-354
        ArenaBvh<T> old;
        std::swap(old, arena);
        arena.reset();
        arena.begin_edit();
        layout = arena.layout;
        nodes = FreeList{};
        nodes.end = 1;
        prims = FreeList{};
        std::vector<Chunk*> placed;
        for (auto& kv : chunks)
            if (!kv.second.nodes.none()) placed.push_back(&kv.second);
        std::stable_sort(placed.begin(), placed.end(), [](Chunk* a, Chunk* b) { return a->prims.lo < b->prims.lo; });
        for (Chunk* c : placed) {
            size_t na = nodes.take(c->nodes.size()), pa = prims.take(c->prims.size());
            arena.write_part(old.b, c->nodes, c->prims, na, pa);
            c->nodes = Span{na, na + c->nodes.size()};
            c->prims = Span{pa, pa + c->prims.size()};
        }
        stats.compacted = 1;
    }
    // scene_cache.rs:281-336.
    void finish(Bvh<T>&& vol, ArenaBvh<T>& arena) {
        for (auto it = chunks.begin(); it != chunks.end();) {
            if (it->second.used != generation) {
                nodes.give(it->second.nodes);
                prims.give(it->second.prims);
                it = chunks.erase(it);
            } else {
                ++it;
            }
        }
        nodes.give(top);
        top = Span{};
        nodes.give(vol_nodes);
        prims.give(vol_prims);
        vol_nodes = vol_prims = Span{};
        auto live = [](const FreeList& f) { return f.end - f.holes(); };
        if (prims.holes() > live(prims) / 2 + (1u << 14) || nodes.holes() > live(nodes) / 2 + (1u << 14)) compact(arena);
        auto place = [&](const Bvh<T>& bvh, Span& nr, Span& pr) {
            size_t n = bvh.nodes.size(), p = bvh.simplices.size();
            size_t na = nodes.take(n), pa = prims.take(p);
            arena.write_part(bvh, Span{0, n}, Span{0, p}, na, pa);
            nr = Span{na, na + n};
            pr = Span{pa, pa + p};
        };
        std::vector<TopItem<T>> items;
        for (const CacheChunkId& id : order) {
            Chunk& c = chunks[id];
            if (c.fresh) {
                place(*c.fresh, c.nodes, c.prims);
                c.bounds = c.fresh->nodes.empty() ? Aabb<T>{} : c.fresh->nodes[0].aabb;
                c.fresh.reset();
            }
            if (!c.nodes.none()) items.push_back({c.bounds, (uint32_t)c.nodes.lo, (T)c.prims.size()});
        }
        if (!vol.nodes.empty()) {
            place(vol, vol_nodes, vol_prims);
            items.push_back({vol.nodes[0].aabb, (uint32_t)vol_nodes.lo, (T)vol.simplices.size()});
        }
        if (items.empty()) {
            BvhNode<T> z = nothing<T>();
            arena.write_nodes(0, &z, 1);
        } else if (items.size() == 1) {
            BvhNode<T> r = arena.b.nodes[items[0].root];
            arena.write_nodes(0, &r, 1);
        } else {
            size_t base = nodes.take(items.size() - 2);
            top = Span{base, base + items.size() - 2};
            std::vector<BvhNode<T>> tree;
            top_tree_rec(items, 0, items.size(), (uint32_t)base, tree);
            arena.write_nodes(0, tree.data(), 1);
            arena.write_nodes(base, tree.data() + 1, tree.size() - 1);
        }
        stats.arena_simplices = prims.end;
    }
};

// A simplex from its packed hot and cold records and its box (gpu.rs:44-92 layouts).
inline Simplex<float> simplex_from_packed(const PGeom& g, const PAttr& a, const float* box8) {
    auto v4 = [](const float* p) { return V4<float>(p[0], p[1], p[2], p[3]); };
    Simplex<float> s;
    s.g.v0 = v4(g.v0); s.g.n = v4(g.n); s.g.b1 = v4(g.b1); s.g.b2 = v4(g.b2); s.g.b3 = v4(g.b3);
    for (int k = 0; k < 4; ++k) {
        s.uv_u[k] = a.uv_u[k]; s.uv_v[k] = a.uv_v[k];
        s.tri_bary[k] = V3<float>(a.tb_x[k], a.tb_y[k], a.tb_z[k]);
        s.tau[k] = a.tau[k]; s.grad_u[k] = a.grad_u[k]; s.grad_v[k] = a.grad_v[k];
        s.decided_at[k] = a.decided_at[k];
    }
    s.normal = v4(a.normal);
    s.four_vel = v4(a.four_vel);
    s.uvs_u = a.misc[0];
    s.uvs_v = a.misc[1];
    std::memcpy(&s.material_id, &a.misc[2], 4);
    s.aabb.min = v4(box8);
    s.aabb.max = v4(box8 + 4);
    return s;
}

}  // namespace orc
