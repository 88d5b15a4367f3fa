// The scene cache over a device arena: SceneCache (dynamic/scene_cache.rs:120-356) with Bvh4D's
// arena edits (bvh4d.rs:168-215 reset_arena / write_part / write_nodes, 583-591 put; top_tree,
// 593-644, in csrc/host/top_tree.cpp), where the arena is the scene's own device arrays.
//
// The bookkeeping runs on the host as the reference's does (first-fit free lists, chunk keys, the
// compaction rule, the tree over the chunks' roots over a few hundred boxes); everything that
// touches simplices runs on the device: a snapshot's new chunks are extruded (sr_extrude.cu) and
// built (sr_build.cu) together as one forest, and every write_part is a copy that moves the
// chunk's links (one launch for all of a snapshot's chunks). The arrays' contents, free room
// included, are the reference arena's byte for byte.
//
// Differences of form, not of result: the reference writes each new chunk into the arena as it
// makes the snapshot; here the scene at the index keeps rendering the previous snapshot until
// sr_arena_finish writes them all. A chunk's key holds the mesh's contents where the reference
// holds a 64-bit hash of them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "../../../include/specrel_scene.h"
#include "sr_build.h"
#include "sr_engine.h"

namespace sre {

namespace {

struct Rng {
    size_t start = 0, end = 0;
    size_t len() const { return end - start; }
    bool empty() const { return end <= start; }
};

// Free ranges of an arena array, first fit (Space, scene_cache.rs:72-115).
struct Space {
    std::vector<Rng> free;  // sorted, disjoint, never adjacent, all before `end`
    size_t end = 0;

    size_t alloc(size_t n) {
        for (size_t k = 0; k < free.size(); ++k)
            if (free[k].len() >= n) {
                const size_t at = free[k].start;
                free[k].start += n;
                if (free[k].empty()) free.erase(free.begin() + k);
                return at;
            }
        end += n;
        return end - n;
    }
    void release(Rng r) {
        if (r.empty()) return;
        size_t k = std::lower_bound(free.begin(), free.end(), r, [](const Rng& f, const Rng& x) { return f.start < x.start; }) -
                   free.begin();
        free.insert(free.begin() + k, r);
        if (k + 1 < free.size() && free[k].end == free[k + 1].start) {
            free[k].end = free[k + 1].end;
            free.erase(free.begin() + k + 1);
        }
        if (k > 0 && free[k - 1].end == free[k].start) {
            free[k - 1].end = free[k].end;
            free.erase(free.begin() + k);
        }
        if (!free.empty() && free.back().end == end) {
            end = free.back().start;
            free.pop_back();
        }
    }
    size_t holes() const {
        size_t h = 0;
        for (const Rng& r : free) h += r.len();
        return h;
    }
};

struct ChunkId {
    uint32_t kind, player;
    uint64_t id;
    int64_t index;
    bool operator<(const ChunkId& o) const {
        if (kind != o.kind) return kind < o.kind;
        if (player != o.player) return player < o.player;
        if (id != o.id) return id < o.id;
        return index < o.index;
    }
};

struct Chunk {
    std::vector<uint32_t> key;
    Rng nodes, prims;        // where it is in the arena (empty: nowhere yet)
    float lo[4], hi[4];      // its root's box
    uint32_t depth = 0, max_leaf = 0;
    int fresh = -1;          // this snapshot's new chunk number, until written
    bool made = false;       // made afresh this snapshot (not reused), until written
    uint64_t used = 0;       // the snapshot that last used it
};

// A new chunk's inputs, kept until sr_arena_finish builds them.
struct NewTube {
    std::vector<float> verts;
    std::vector<SrTubeTriangle> tris;
    std::vector<SrTubeSample> samples;
    std::vector<float> decided;
    bool has_decided = false;
    uint32_t material = 0;
};
struct NewPrims {
    std::vector<float> boxes;
    std::vector<SrGpuGeom> geoms;
    std::vector<SrGpuAttr> attrs;
};
struct NewChunk {
    bool tube;
    size_t at;  // index into tubes / prims
};

constexpr float CHUNK_T = 1.0f;  // scene_cache.rs:32
constexpr size_t COMPACT_SLACK = 1u << 14;

// One copy of write_part: a chunk's nodes and records to their arena slots, links moved.
struct CopyJob {
    uint32_t src_node, dst_node, n_nodes;
    uint32_t src_prim, dst_prim, n_prims;
};

__global__ void k_arena_copy(const CopyJob* jobs, const SrGpuNode* sn, const float4* sg, const float4* sa,
                             SrGpuNode* dn, float4* dg, float4* da) {
    const CopyJob jb = jobs[blockIdx.y];
    const uint32_t step = gridDim.x * blockDim.x, t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t mn = jb.dst_node - jb.src_node, mp = jb.dst_prim - jb.src_prim;  // wrapping, as moved()
    for (uint32_t j = t0; j < jb.n_nodes; j += step) {
        SrGpuNode nd = sn[jb.src_node + j];
        if (nd.count > 0) {
            nd.right_or_first += mp;
        } else {
            nd.left += mn;
            nd.right_or_first += mn;
        }
        dn[jb.dst_node + j] = nd;
    }
    for (uint32_t j = t0; j < 5u * jb.n_prims; j += step) dg[5ull * jb.dst_prim + j] = sg[5ull * jb.src_prim + j];
    for (uint32_t j = t0; j < 12u * jb.n_prims; j += step) da[12ull * jb.dst_prim + j] = sa[12ull * jb.src_prim + j];
}

__global__ void k_gather_nodes(const SrGpuNode* nodes, const uint32_t* at, uint32_t n, SrGpuNode* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = nodes[at[i]];
}

cudaError_t run_jobs(const std::vector<CopyJob>& jobs, const SrGpuNode* sn, const SrGpuGeom* sg, const SrGpuAttr* sa,
                     SrGpuNode* dn, SrGpuGeom* dg, SrGpuAttr* da, cudaStream_t st) {
    if (jobs.empty()) return cudaSuccess;
    uint32_t most = 1;
    for (const CopyJob& j : jobs) most = std::max({most, j.n_nodes, 12u * j.n_prims});
    CopyJob* dj = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&dj), jobs.size() * sizeof(CopyJob), st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(CopyJob), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const uint32_t gx = std::min<uint32_t>((most + 255) / 256, 64);
        k_arena_copy<<<dim3(gx, (uint32_t)jobs.size()), 256, 0, st>>>(
            dj, sn, reinterpret_cast<const float4*>(sg), reinterpret_cast<const float4*>(sa), dn,
            reinterpret_cast<float4*>(dg), reinterpret_cast<float4*>(da));
        e = cudaGetLastError();
    }
    cudaFreeAsync(dj, st);
    return e;
}

// An empty box and the node over nothing (BvhNode4D::NOTHING, bvh4d.rs:31).
SrGpuNode nothing_node() {
    SrGpuNode n{};
    for (int k = 0; k < 4; ++k) { n.min[k] = INFINITY; n.max[k] = -INFINITY; }
    return n;
}

struct Item {
    float box[8];  // min (t, x, y, z), max
    uint32_t root;
    float weight;
    uint32_t depth;  // the chunk's own depth
};

}  // namespace

// The cache of one scene index (SceneCache's state) and the lengths of its arena's arrays.
struct ArenaCache {
    std::map<ChunkId, Chunk> chunks;
    std::vector<ChunkId> order;  // this snapshot's chunks, in the order they were used
    uint64_t generation = 0;
    Space nodes, prims;
    Rng top, vol_nodes, vol_prims;
    SrArenaStats stats{};
    bool reset_pending = true;  // the arrays are not this cache's arena yet (reset_arena at finish)
    bool open = false;          // between sr_arena_begin and sr_arena_finish
    size_t len_nodes = 0, len_prims = 0;
    std::vector<NewChunk> fresh;
    std::vector<NewTube> tubes;
    std::vector<NewPrims> prims_in;
    std::vector<uint32_t> key;  // scratch
    std::map<std::vector<uint32_t>, uint32_t> mesh_ids;  // each distinct mesh's bits, interned
    uint32_t next_mesh_id = 0;  // never reused, so a key made before the map was cleared stays distinct
    // What this snapshot changed before anything is written, to undo a snapshot that fails or is
    // never finished: the free lists at sr_arena_begin and the chunks replaced since (whether they
    // existed, and their state then).
    Space nodes0, prims0;
    std::map<ChunkId, std::pair<bool, Chunk>> journal;

    ArenaCache() { nodes.end = 1; }  // node 0 is the root

    void rollback() {
        for (auto& kv : journal) {
            if (kv.second.first) chunks[kv.first] = std::move(kv.second.second);
            else chunks.erase(kv.first);
        }
        journal.clear();
        nodes = nodes0;
        prims = prims0;
        for (auto& kv : chunks) {
            kv.second.fresh = -1;
            kv.second.made = false;
        }
    }

    // SceneCache::reuse (scene_cache.rs:168-192). Returns 1 reused, 0 not, -1 used twice.
    int reuse(const ChunkId& id, const std::vector<uint32_t>& k) {
        auto found = chunks.find(id);
        const bool existed = found != chunks.end();
        Chunk& c = existed ? found->second : chunks[id];
        if (c.used == generation) return -1;
        const bool reused = c.used != 0 && c.key == k;
        if (!reused && !journal.count(id)) journal.emplace(id, std::make_pair(existed, existed ? c : Chunk{}));
        if (reused) {
            stats.chunks_reused += 1;
            stats.simplices_reused += c.prims.len();
        } else {
            nodes.release(c.nodes);
            prims.release(c.prims);
            c.nodes = Rng{};
            c.prims = Rng{};
            c.key = k;
            c.fresh = -1;
            c.made = true;
        }
        c.used = generation;
        order.push_back(id);
        return reused ? 1 : 0;
    }
};

}  // namespace sre

using namespace sre;

namespace {

// Scratch from the stream-ordered pool, freed in stream order.
struct TBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~TBuf() { if (p) cudaFreeAsync(p, st); }
    cudaError_t alloc(size_t n, cudaStream_t s) {
        st = s;
        return cudaMallocAsync(&p, std::max<size_t>(n, 16), s);
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

sr_status open_cache(sr_ctx* ctx, uint32_t idx, ArenaCache** out) {
    if (!ctx) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->arena || !ctx->scenes[idx]->arena->open)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "no snapshot begun at this index (sr_arena_begin)");
    *out = ctx->scenes[idx]->arena.get();
    return SR_OK;
}

// Grows a device array to `n` bytes keeping its first `keep` bytes.
cudaError_t grow_keep(DevBuf& b, size_t n, size_t keep, cudaStream_t st) {
    if (n <= b.bytes && b.p) return cudaSuccess;
    size_t cap = std::max(n, b.bytes + b.bytes / 2);
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, cap);
    if (e != cudaSuccess) return e;
    if (keep && b.p) e = cudaMemcpyAsync(p, b.p, keep, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(p);
        return e;
    }
    if (b.p) cudaFree(b.p);
    b.p = p;
    b.bytes = cap;
    return cudaSuccess;
}

void push_sample_key(std::vector<uint32_t>& k, const SrTubeSample& s) {  // push_sample, scene_cache.rs:358-366
    auto put = [&](const float* v, int n) {
        for (int i = 0; i < n; ++i) {
            uint32_t u;
            std::memcpy(&u, &v[i], 4);
            k.push_back(u);
        }
    };
    put(s.center, 4);
    put(&s.proper_time, 1);
    put(s.phi, 3);
    put(s.accel, 3);
    for (int e = 0; e < 4; ++e) put(s.tetrad[e], 4);
}

}  // namespace

extern "C" {

sr_status sr_arena_begin(sr_ctx* ctx, uint32_t idx) {
    if (!ctx) return SR_ERR_INVALID_ARGUMENT;
    if (idx > 4096) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "scene index too large");
    if (ctx->scenes.size() <= idx) ctx->scenes.resize(idx + 1);
    if (!ctx->scenes[idx]) ctx->scenes[idx] = std::make_unique<SceneSlot>();
    SceneSlot& s = *ctx->scenes[idx];
    if (!s.arena) s.arena = std::make_shared<ArenaCache>();  // a fresh layout (SceneCache::begin)
    ArenaCache& a = *s.arena;
    if (a.open) a.rollback();  // a snapshot begun and never finished is undone
    a.generation += 1;
    a.order.clear();
    a.stats = SrArenaStats{};
    a.fresh.clear();
    a.tubes.clear();
    a.prims_in.clear();
    a.journal.clear();
    a.nodes0 = a.nodes;
    a.prims0 = a.prims;
    a.open = true;
    return SR_OK;
}

sr_status sr_arena_tube(sr_ctx* ctx, uint32_t idx, SrArenaPart part, const SrTube* tube) {
    ArenaCache* ap = nullptr;
    sr_status r = open_cache(ctx, idx, &ap);
    if (r != SR_OK) return r;
    if (!tube) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "tube is null");
    const SrTube& t = *tube;
    if ((t.num_vertices && !t.vertices) || (t.num_triangles && !t.triangles) || (t.num_samples && !t.samples))
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "tube: null array");
    for (uint32_t i = 0; i < t.num_triangles; ++i)
        for (int k = 0; k < 3; ++k)
            if (t.triangles[i].idx[k] >= t.num_vertices) return fail(ctx, SR_ERR_BAD_SCENE, "tube: vertex index out of range");
    if ((uint64_t)t.num_samples * t.num_vertices > 0xFFFFFFFFull || (uint64_t)t.num_samples * t.num_triangles > 0x3FFFFFFFull)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "tube: too many samples");
    ArenaCache& a = *ap;
    if (t.num_samples < 2) return SR_OK;
    // The mesh's bits stand for mesh_fingerprint (scene_cache.rs:368-380): interned once, the
    // chunks' keys hold the mesh's id (equal ids, equal meshes).
    std::vector<uint32_t> mesh;
    mesh.push_back(t.num_vertices);
    mesh.push_back(t.num_triangles);
    for (uint32_t i = 0; i < 3 * t.num_vertices; ++i) {
        uint32_t u;
        std::memcpy(&u, &t.vertices[i], 4);
        mesh.push_back(u);
    }
    for (uint32_t i = 0; i < t.num_triangles; ++i) {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(&t.triangles[i]);
        mesh.insert(mesh.end(), w, w + sizeof(SrTubeTriangle) / 4);
    }
    auto found = a.mesh_ids.find(mesh);
    if (found == a.mesh_ids.end()) {
        if (a.mesh_ids.size() >= 1024) a.mesh_ids.clear();  // bounded: chunks of forgotten meshes are rebuilt
        found = a.mesh_ids.emplace(std::move(mesh), a.next_mesh_id++).first;
    }
    const uint32_t mesh_id = found->second;
    auto bucket = [&](uint32_t i) -> int64_t {  // (center.t / CHUNK_T).floor() as i64
        const double f = std::floor((double)(t.samples[i].center[0] / CHUNK_T));
        if (std::isnan(f)) return 0;
        if (f >= 9.2233720368547758e18) return INT64_MAX;
        if (f <= -9.2233720368547758e18) return INT64_MIN;
        return (int64_t)f;
    };
    const ChunkId base{part.kind, part.player, part.id, 0};
    uint32_t first = 0;
    while (first < t.num_samples - 1) {  // SceneCache::tube (scene_cache.rs:203-248)
        const int64_t b = bucket(first);
        uint32_t end = first + 1;
        while (end < t.num_samples - 1 && bucket(end) == b) ++end;
        std::vector<uint32_t>& key = a.key;
        key.clear();
        key.push_back(t.material);
        key.push_back(t.decided_at ? 1u : 0u);
        key.push_back(mesh_id);
        for (uint32_t i = first; i <= end; ++i) push_sample_key(key, t.samples[i]);
        if (t.decided_at)
            for (uint32_t i = first; i <= end; ++i) {
                uint32_t u;
                std::memcpy(&u, &t.decided_at[i], 4);
                key.push_back(u);
            }
        ChunkId id = base;
        id.index = b;
        const int reused = a.reuse(id, key);
        if (reused < 0) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "a chunk was made twice in one snapshot");
        if (!reused) {
            NewTube nt;
            nt.verts.assign(t.vertices, t.vertices + 3 * t.num_vertices);
            nt.tris.assign(t.triangles, t.triangles + t.num_triangles);
            nt.samples.assign(t.samples + first, t.samples + end + 1);
            nt.has_decided = t.decided_at != nullptr;
            if (t.decided_at) nt.decided.assign(t.decided_at + first, t.decided_at + end + 1);
            nt.material = t.material;
            a.chunks[id].fresh = (int)a.fresh.size();
            a.fresh.push_back({true, a.tubes.size()});
            a.tubes.push_back(std::move(nt));
        }
        first = end;
    }
    return SR_OK;
}

sr_status sr_arena_reuse(sr_ctx* ctx, uint32_t idx, SrArenaPart part, int64_t index, const uint32_t* key,
                         uint32_t key_len, int32_t* reused) {
    ArenaCache* ap = nullptr;
    sr_status r = open_cache(ctx, idx, &ap);
    if (r != SR_OK) return r;
    if (!reused || (key_len && !key)) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "null key or result");
    std::vector<uint32_t> k(key, key + key_len);
    const int u = ap->reuse(ChunkId{part.kind, part.player, part.id, index}, k);
    if (u < 0) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "a chunk was made twice in one snapshot");
    *reused = u;
    return SR_OK;
}

sr_status sr_arena_install(sr_ctx* ctx, uint32_t idx, SrArenaPart part, int64_t index, const float* boxes,
                           const SrGpuGeom* geoms, const SrGpuAttr* attrs, uint32_t n) {
    ArenaCache* ap = nullptr;
    sr_status r = open_cache(ctx, idx, &ap);
    if (r != SR_OK) return r;
    if (n && (!boxes || !geoms || !attrs)) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "null simplex arrays");
    ArenaCache& a = *ap;
    auto it = a.chunks.find(ChunkId{part.kind, part.player, part.id, index});
    if (it == a.chunks.end() || it->second.used != a.generation || !it->second.nodes.empty() || it->second.fresh >= 0)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "install follows sr_arena_reuse answering 0, once");
    NewPrims p;
    p.boxes.assign(boxes, boxes + 8ull * n);
    p.geoms.assign(geoms, geoms + n);
    p.attrs.assign(attrs, attrs + n);
    it->second.fresh = (int)a.fresh.size();
    a.fresh.push_back({false, a.prims_in.size()});
    a.prims_in.push_back(std::move(p));
    return SR_OK;
}

sr_status sr_arena_finish(sr_ctx* ctx, uint32_t idx, const SrBuildDesc* d, SrArenaStats* stats_out) {
    ArenaCache* ap = nullptr;
    sr_status r = open_cache(ctx, idx, &ap);
    if (r != SR_OK) return r;
    if (!d) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "desc is null");
    const uint32_t nvol = d->num_prims;
    if (nvol && (!d->boxes || !d->geoms || !d->attrs)) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "null volatile arrays");
    r = check_build_desc(ctx, d, nvol ? d->attrs : nullptr, nvol);
    if (r != SR_OK) return r;
    ArenaCache& a = *ap;
    for (const NewTube& t : a.tubes)
        if (t.material >= d->num_materials) return fail(ctx, SR_ERR_BAD_SCENE, "tube material id out of range");
    for (const NewPrims& p : a.prims_in)
        for (const SrGpuAttr& at : p.attrs) {  // the installed simplices' material ids
            uint32_t m;
            std::memcpy(&m, &at.misc[2], 4);
            if (m >= d->num_materials) return fail(ctx, SR_ERR_BAD_SCENE, "an installed simplex's material id is out of range");
        }
    CK(cudaSetDevice(ctx->device), "set device");
    cudaStream_t st = ctx->stream;
    SceneSlot& s = *ctx->scenes[idx];
    const bool was_live = s.present;  // its launch tuning (sr_set_tuning, sr_autotune) is kept
    a.open = false;
    // Until the arrays are written, a failure undoes the snapshot (the scene and its cache are as
    // they were); after, it leaves no scene at the index.
    struct Abandon {
        SceneSlot* s;
        ArenaCache* a;
        bool armed = false, done = false;
        ~Abandon() {
            if (done) return;
            if (armed) {
                s->present = false;
                s->arena.reset();
            } else {
                a->rollback();
            }
        }
    } abandon{&s, &a};
    std::shared_ptr<ArenaCache> hold = s.arena;  // `a` outlives the slot's reference on failure
    CK(keep_build_pool(), "memory pool");

    // 1. The new chunks and the volatile part as one forest, built on the device.
    std::vector<SrTube> tv(a.tubes.size());
    for (size_t i = 0; i < a.tubes.size(); ++i) {
        const NewTube& t = a.tubes[i];
        tv[i] = SrTube{t.verts.data(), (uint32_t)(t.verts.size() / 3), (uint32_t)t.tris.size(), t.tris.data(),
                       t.samples.data(), (uint32_t)t.samples.size(), t.material, t.has_decided ? t.decided.data() : nullptr};
    }
    ExtrudeOut ex{};
    std::vector<uint32_t> tube_first(tv.size() + 1, 0);
    struct FreeEx {
        ExtrudeOut* x;
        cudaStream_t st;
        ~FreeEx() {
            if (x->geoms) cudaFreeAsync(x->geoms, st);
            if (x->attrs) cudaFreeAsync(x->attrs, st);
            if (x->boxes) cudaFreeAsync(x->boxes, st);
        }
    } free_ex{&ex, st};
    if (!tv.empty()) CK(gpu_extrude(tv.data(), (uint32_t)tv.size(), &ex, st, tube_first.data()), "extrude");
    a.stats.rindler_crossed = ex.rindler_bad;
    std::vector<GpuSegment> segs;
    std::vector<size_t> seg_of_fresh(a.fresh.size());
    uint64_t total = ex.num_prims;
    for (size_t i = 0; i < a.tubes.size(); ++i) segs.push_back({tube_first[i], tube_first[i + 1] - tube_first[i]});
    for (size_t i = 0; i < a.prims_in.size(); ++i) {
        const uint32_t c = (uint32_t)a.prims_in[i].geoms.size();
        segs.push_back({(uint32_t)total, c});
        total += c;
    }
    for (size_t f = 0; f < a.fresh.size(); ++f)
        seg_of_fresh[f] = a.fresh[f].tube ? a.fresh[f].at : a.tubes.size() + a.fresh[f].at;
    const size_t vol_seg = segs.size();
    segs.push_back({(uint32_t)total, nvol});
    total += nvol;
    if (total >= 0x7FFFFFFFull) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "too many new simplices in one snapshot");
    const uint32_t n = (uint32_t)total;
    TBuf box, gin, ain, fnodes, forder, gl, al;
    std::vector<GpuTreeInfo> tree(segs.size());
    std::vector<SrGpuNode> roots(segs.size(), nothing_node());
    if (n) {
        CK(box.alloc((size_t)n * 32, st), "alloc boxes");
        CK(gin.alloc((size_t)n * sizeof(SrGpuGeom), st), "alloc geoms");
        CK(ain.alloc((size_t)n * sizeof(SrGpuAttr), st), "alloc attrs");
        if (ex.num_prims) {
            CK(cudaMemcpyAsync(box.p, ex.boxes, (size_t)ex.num_prims * 32, cudaMemcpyDeviceToDevice, st), "copy boxes");
            CK(cudaMemcpyAsync(gin.p, ex.geoms, (size_t)ex.num_prims * sizeof(SrGpuGeom), cudaMemcpyDeviceToDevice, st),
               "copy geoms");
            CK(cudaMemcpyAsync(ain.p, ex.attrs, (size_t)ex.num_prims * sizeof(SrGpuAttr), cudaMemcpyDeviceToDevice, st),
               "copy attrs");
        }
        auto upload = [&](uint32_t at, const float* bx, const SrGpuGeom* g, const SrGpuAttr* at_, uint32_t c) -> cudaError_t {
            if (!c) return cudaSuccess;
            cudaError_t e = cudaMemcpyAsync(box.as<float4>() + 2ull * at, bx, (size_t)c * 32, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(gin.as<SrGpuGeom>() + at, g, (size_t)c * sizeof(SrGpuGeom), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ain.as<SrGpuAttr>() + at, at_, (size_t)c * sizeof(SrGpuAttr), cudaMemcpyHostToDevice, st);
            return e;
        };
        for (size_t i = 0; i < a.prims_in.size(); ++i) {
            const NewPrims& p = a.prims_in[i];
            CK(upload(segs[a.tubes.size() + i].start, p.boxes.data(), p.geoms.data(), p.attrs.data(),
                      (uint32_t)p.geoms.size()),
               "upload simplices");
        }
        CK(upload(segs[vol_seg].start, d->boxes, d->geoms, d->attrs, nvol), "upload volatile simplices");
        CK(fnodes.alloc((size_t)2 * n * sizeof(SrGpuNode), st), "alloc forest");
        CK(forder.alloc((size_t)n * 4, st), "alloc order");
        GpuBuildInfo info{};
        CK(gpu_bvh_build_forest(box.as<float4>(), n, segs.data(), (uint32_t)segs.size(), fnodes.as<SrGpuNode>(),
                                forder.as<uint32_t>(), tree.data(), &info, st),
           "build chunks");
        if (info.unsupported)
            return fail(ctx, SR_ERR_UNSUPPORTED,
                        "a split left one side empty: the reference selects by median there");
        CK(gl.alloc((size_t)n * sizeof(SrGpuGeom), st), "alloc geoms");
        CK(al.alloc((size_t)n * sizeof(SrGpuAttr), st), "alloc attrs");
        CK(gpu_gather_records(forder.as<uint32_t>(), n, gin.as<SrGpuGeom>(), ain.as<SrGpuAttr>(), gl.as<SrGpuGeom>(),
                              al.as<SrGpuAttr>(), st),
           "leaf order");
        std::vector<uint32_t> at;
        for (const GpuTreeInfo& t : tree) at.push_back(t.node_base);
        TBuf dat, droots;
        CK(dat.alloc(at.size() * 4, st), "alloc");
        CK(droots.alloc(at.size() * sizeof(SrGpuNode), st), "alloc");
        CK(cudaMemcpyAsync(dat.p, at.data(), at.size() * 4, cudaMemcpyHostToDevice, st), "upload");
        k_gather_nodes<<<((uint32_t)at.size() + 127) / 128, 128, 0, st>>>(fnodes.as<SrGpuNode>(), dat.as<uint32_t>(),
                                                                           (uint32_t)at.size(), droots.as<SrGpuNode>());
        CK(cudaGetLastError(), "gather roots");
        CK(cudaMemcpyAsync(roots.data(), droots.p, at.size() * sizeof(SrGpuNode), cudaMemcpyDeviceToHost, st), "read roots");
        CK(cudaStreamSynchronize(st), "build sync");
        for (size_t i = 0; i < segs.size(); ++i)
            if (tree[i].num_nodes == 0) roots[i] = nothing_node();
    }

    // 2. SceneCache::finish (scene_cache.rs:281-336): drop unused chunks, free the old top tree and
    // volatile part, compact if the free room is too large, place the new chunks, the tree.
    abandon.armed = true;
    const uint64_t gen = a.generation;
    for (auto it = a.chunks.begin(); it != a.chunks.end();) {
        if (it->second.used != gen) {
            a.nodes.release(it->second.nodes);
            a.prims.release(it->second.prims);
            it = a.chunks.erase(it);
        } else {
            ++it;
        }
    }
    a.nodes.release(a.top);
    a.top = Rng{};
    a.nodes.release(a.vol_nodes);
    a.prims.release(a.vol_prims);
    a.vol_nodes = Rng{};
    a.vol_prims = Rng{};

    if (a.reset_pending) {  // reset_arena (bvh4d.rs:170-179): node 0 over nothing
        const SrGpuNode z = nothing_node();
        CK(grow_keep(s.nodes, sizeof(SrGpuNode), 0, st), "alloc nodes");
        CK(cudaMemcpyAsync(s.nodes.p, &z, sizeof(z), cudaMemcpyHostToDevice, st), "reset arena");
        a.len_nodes = 1;
        a.len_prims = 0;
        a.reset_pending = false;
    }
    auto live = [](const Space& sp) { return sp.end - sp.holes(); };
    if (a.prims.holes() > live(a.prims) / 2 + COMPACT_SLACK || a.nodes.holes() > live(a.nodes) / 2 + COMPACT_SLACK) {
        // compact (scene_cache.rs:338-354): the placed chunks moved together into a fresh layout.
        std::vector<Chunk*> placed;
        for (auto& kv : a.chunks)
            if (!kv.second.nodes.empty()) placed.push_back(&kv.second);
        std::sort(placed.begin(), placed.end(), [](const Chunk* x, const Chunk* y) { return x->prims.start < y->prims.start; });
        a.nodes = Space{};
        a.nodes.end = 1;
        a.prims = Space{};
        std::vector<CopyJob> jobs;
        for (Chunk* c : placed) {
            const size_t na = a.nodes.alloc(c->nodes.len()), pa = a.prims.alloc(c->prims.len());
            jobs.push_back({(uint32_t)c->nodes.start, (uint32_t)na, (uint32_t)c->nodes.len(), (uint32_t)c->prims.start,
                            (uint32_t)pa, (uint32_t)c->prims.len()});
            c->nodes = Rng{na, na + c->nodes.len()};
            c->prims = Rng{pa, pa + c->prims.len()};
        }
        DevBuf nn, ng, na;
        CK(nn.ensure(std::max<size_t>(a.nodes.end, 1) * sizeof(SrGpuNode)), "alloc arena");
        CK(ng.ensure(std::max<size_t>(a.prims.end, 1) * sizeof(SrGpuGeom)), "alloc arena");
        CK(na.ensure(std::max<size_t>(a.prims.end, 1) * sizeof(SrGpuAttr)), "alloc arena");
        const SrGpuNode z = nothing_node();
        CK(cudaMemcpyAsync(nn.p, &z, sizeof(z), cudaMemcpyHostToDevice, st), "reset arena");
        CK(run_jobs(jobs, s.nodes.as<SrGpuNode>(), s.geoms.as<SrGpuGeom>(), s.attrs.as<SrGpuAttr>(), nn.as<SrGpuNode>(),
                    ng.as<SrGpuGeom>(), na.as<SrGpuAttr>(), st),
           "compact");
        CK(cudaStreamSynchronize(st), "compact sync");
        std::swap(s.nodes.p, nn.p);
        std::swap(s.nodes.bytes, nn.bytes);
        std::swap(s.geoms.p, ng.p);
        std::swap(s.geoms.bytes, ng.bytes);
        std::swap(s.attrs.p, na.p);
        std::swap(s.attrs.bytes, na.bytes);
        a.len_nodes = a.nodes.end;
        a.len_prims = a.prims.end;
        a.stats.compacted = 1;
    }

    // Placement of this snapshot's new chunks (in the order they were used) and of the volatile
    // part; then every write at once.
    std::vector<CopyJob> jobs;
    std::vector<Item> items;
    uint32_t max_leaf = 0;
    size_t need_nodes = a.len_nodes, need_prims = a.len_prims;
    auto place = [&](size_t sg, Rng& nr, Rng& pr) {
        const GpuTreeInfo& t = tree[sg];
        const size_t nn = t.num_nodes, np = segs[sg].count;
        const size_t na = a.nodes.alloc(nn), pa = a.prims.alloc(np);
        if (nn) jobs.push_back({t.node_base, (uint32_t)na, (uint32_t)nn, segs[sg].start, (uint32_t)pa, (uint32_t)np});
        nr = Rng{na, na + nn};
        pr = Rng{pa, pa + np};
        need_nodes = std::max(need_nodes, na + nn);
        need_prims = std::max(need_prims, pa + np);
    };
    for (const ChunkId& id : a.order) {
        Chunk& c = a.chunks[id];
        if (c.made) {  // SceneCache::install; a chunk never installed is a build over nothing
            a.stats.chunks_built += 1;
            if (c.fresh >= 0) {
                const size_t sg = seg_of_fresh[c.fresh];
                place(sg, c.nodes, c.prims);
                for (int k = 0; k < 4; ++k) { c.lo[k] = roots[sg].min[k]; c.hi[k] = roots[sg].max[k]; }
                c.depth = tree[sg].depth;
                c.max_leaf = tree[sg].max_leaf;
                a.stats.simplices_built += segs[sg].count;
            }
            c.fresh = -1;
            c.made = false;
        }
        if (!c.nodes.empty()) {
            Item it{};
            std::copy(c.lo, c.lo + 4, it.box);
            std::copy(c.hi, c.hi + 4, it.box + 4);
            it.root = (uint32_t)c.nodes.start;
            it.weight = (float)c.prims.len();
            it.depth = c.depth;
            items.push_back(it);
            max_leaf = std::max(max_leaf, c.max_leaf);
        }
    }
    if (tree[vol_seg].num_nodes > 0) {
        place(vol_seg, a.vol_nodes, a.vol_prims);
        Item it{};
        for (int k = 0; k < 4; ++k) { it.box[k] = roots[vol_seg].min[k]; it.box[4 + k] = roots[vol_seg].max[k]; }
        it.root = (uint32_t)a.vol_nodes.start;
        it.weight = (float)nvol;
        it.depth = tree[vol_seg].depth;
        items.push_back(it);
        max_leaf = std::max(max_leaf, tree[vol_seg].max_leaf);
    }
    std::vector<SrGpuNode> top_nodes;
    size_t top_base = 0;
    uint32_t depth = 1;
    if (items.size() >= 2) {  // top_tree (bvh4d.rs:593-644; csrc/host/top_tree.cpp)
        top_base = a.nodes.alloc(items.size() - 2);
        a.top = Rng{top_base, top_base + items.size() - 2};
        need_nodes = std::max(need_nodes, a.top.end);
        const size_t ni = items.size();
        std::vector<float> bx(8 * ni), w(ni);
        std::vector<uint32_t> rt(ni), dp(ni);
        for (size_t i = 0; i < ni; ++i) {
            std::copy(items[i].box, items[i].box + 8, &bx[8 * i]);
            rt[i] = items[i].root;
            w[i] = items[i].weight;
            dp[i] = items[i].depth;
        }
        top_nodes.resize(ni - 1);
        if (sr_top_tree(bx.data(), rt.data(), w.data(), dp.data(), (uint32_t)ni, (uint32_t)top_base, top_nodes.data(),
                        &depth) != SR_OK)
            return fail(ctx, SR_ERR_INVALID_ARGUMENT, "top tree");
    } else if (items.size() == 1) {
        depth = items[0].depth;
    }
    if (need_nodes > 0xFFFFFFF0ull || need_prims > 0xFFFFFFF0ull)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "the arena outgrew 32-bit indices");
    CK(grow_keep(s.nodes, need_nodes * sizeof(SrGpuNode), a.len_nodes * sizeof(SrGpuNode), st), "grow arena");
    CK(grow_keep(s.geoms, std::max<size_t>(need_prims, 1) * sizeof(SrGpuGeom), a.len_prims * sizeof(SrGpuGeom), st),
       "grow arena");
    CK(grow_keep(s.attrs, std::max<size_t>(need_prims, 1) * sizeof(SrGpuAttr), a.len_prims * sizeof(SrGpuAttr), st),
       "grow arena");
    if (!jobs.empty())
        CK(run_jobs(jobs, fnodes.as<SrGpuNode>(), gl.as<SrGpuGeom>(), al.as<SrGpuAttr>(), s.nodes.as<SrGpuNode>(),
                    s.geoms.as<SrGpuGeom>(), s.attrs.as<SrGpuAttr>(), st),
           "write chunks");
    SrGpuNode* dn = s.nodes.as<SrGpuNode>();
    if (items.empty()) {
        const SrGpuNode z = nothing_node();
        CK(cudaMemcpyAsync(dn, &z, sizeof(z), cudaMemcpyHostToDevice, st), "write root");
    } else if (items.size() == 1) {
        CK(cudaMemcpyAsync(dn, dn + items[0].root, sizeof(SrGpuNode), cudaMemcpyDeviceToDevice, st), "write root");
    } else {
        CK(cudaMemcpyAsync(dn, top_nodes.data(), sizeof(SrGpuNode), cudaMemcpyHostToDevice, st), "write root");
        if (top_nodes.size() > 1)
            CK(cudaMemcpyAsync(dn + top_base, top_nodes.data() + 1, (top_nodes.size() - 1) * sizeof(SrGpuNode),
                               cudaMemcpyHostToDevice, st),
               "write top tree");
    }
    a.len_nodes = need_nodes;
    a.len_prims = need_prims;
    a.stats.arena_simplices = a.prims.end;
    a.stats.num_nodes = (uint32_t)a.len_nodes;
    a.stats.bvh_depth = depth;
    CK(cudaStreamSynchronize(st), "arena sync");

    // 3. The scene goes live: the arrays as the reference's GPU copy of the arena, the node layout.
    r = upload_scene_rest(ctx, s, d);
    if (r != SR_OK) return r;
    s.num_nodes = (uint32_t)a.len_nodes;
    s.num_prims = (uint32_t)a.len_prims;
    s.depth = depth;
    s.has_l2o = false;
    s.empty_tree = items.empty();
    s.rindler_crossed = a.stats.rindler_crossed != 0;
    s.fast.layout = ctx->layout_of(idx);
    CK(fast_build(ctx->fast, s.fast, s.nodes.as<SrGpuNode>(), s.num_nodes, depth, s.num_prims, max_leaf, st),
       "build node layout");
    if (!was_live) s.tuning = fast_default_tuning(ctx->fast);
    a.fresh.clear();
    a.tubes.clear();
    a.prims_in.clear();
    s.present = true;
    a.journal.clear();
    abandon.done = true;
    if (stats_out) *stats_out = a.stats;
    return SR_OK;
}

}  // extern "C"
