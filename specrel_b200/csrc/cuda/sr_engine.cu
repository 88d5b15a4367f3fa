// The C ABI of include/specrel.h: contexts, scene upload (with host-side validation), frame
// buffers and the render entry points. Mirrors GpuRenderer (gpu.rs:432-901): the context owns
// the device copies of every scene, one stream, and the per-resolution frame buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/specrel.h"
#include "../../../include/specrel_scene.h"
#include "sr_build.h"
#include "sr_fast.h"
#include "sr_engine.h"

using namespace srk;
using namespace sre;

namespace {

// Blackbody constants (star.rs:162-180): powi(5) folded in double precision, white-point Planck
// values in f32, as the compiled reference evaluates them.
BBConst make_bb() {
    auto p5 = [](float l) { return (float)std::pow((double)l, 5.0); };
    auto planck = [&](float l, float t) {
        float x = std::fmin(14388.0f / (l * std::fmax(t, 1.0f)), 80.0f);
        return 1.0f / (p5(l) * (std::exp(x) - 1.0f));
    };
    BBConst b;
    b.r5 = p5(0.610f);
    b.g5 = p5(0.550f);
    b.b5 = p5(0.465f);
    b.wr = planck(0.610f, 6504.0f);
    b.wg = planck(0.550f, 6504.0f);
    b.wb = planck(0.465f, 6504.0f);
    return b;
}

SceneDev scene_dev(const sr_ctx* ctx, const SceneSlot& s) {
    SceneDev d{};
    d.nodes = s.nodes.as<SrGpuNode>();
    d.geoms = s.geoms.as<float4>();
    d.attrs = s.attrs.as<float4>();
    d.mats = s.mats.as<float4>();
    d.stars = s.stars.as<float4>();
    d.leaf_to_orig = s.has_l2o ? s.l2o.as<uint32_t>() : nullptr;
    d.tables = ctx->tables.as<uint32_t>();
    d.wide = nullptr;
    d.num_nodes = s.empty_tree ? 0 : s.num_nodes;
    d.num_prims = s.num_prims;
    d.num_mats = s.num_mats;
    d.num_stars = s.num_stars;
    return d;
}

uint32_t max_leaf_of(const SrSceneDesc* d) {
    uint32_t m = 0;
    for (uint32_t i = 0; i < d->num_nodes; ++i) m = std::max(m, d->nodes[i].count);
    return m;
}

sr_status ensure_frame(sr_ctx* ctx, uint32_t w, uint32_t h) {
    Frame& f = ctx->frame;
    if (f.w == w && f.h == h && f.hdr.p) return SR_OK;
    Pyramid p = make_pyramid(w, h);
    CK(f.hdr.ensure((size_t)p.off[SR_BLOOM_LEVELS + 1] * sizeof(float4)), "frame hdr");
    CK(f.rgb.ensure((size_t)w * h * 4), "frame rgb");
    f.pyr = p;
    f.w = w;
    f.h = h;
    return SR_OK;
}

}  // namespace

extern "C" {

sr_status sr_create(int device, sr_ctx** out, char* err, size_t errlen) {
    auto set = [&](const std::string& m) {
        if (err && errlen) { std::strncpy(err, m.c_str(), errlen - 1); err[errlen - 1] = 0; }
    };
    if (!out) { set("out is null"); return SR_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) { set(std::string("no CUDA device: ") + cudaGetErrorString(e)); return SR_ERR_NO_DEVICE; }
    if (device < 0 || device >= n) { set("device index out of range"); return SR_ERR_INVALID_ARGUMENT; }
    auto ctx = std::make_unique<sr_ctx>();
    ctx->device = device;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) { set(cudaGetErrorString(e)); return SR_ERR_CUDA; }
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    ctx->name = std::string(prop.name) + " (CUDA sm_" + std::to_string(prop.major) + std::to_string(prop.minor) + ")";
    if (prop.major < 10) { set("this build targets sm_100a (B200); device is " + ctx->name); return SR_ERR_UNSUPPORTED; }
    if ((e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking)) != cudaSuccess) { set(cudaGetErrorString(e)); return SR_ERR_CUDA; }
    ctx->stream = ctx->own;
    std::vector<uint32_t> tables(SR_GAMMA_LUT_SIZE + 14 * 7);
    sr_tables_build(tables.data());
    if ((e = ctx->tables.ensure(tables.size() * 4)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->tables.p, tables.data(), tables.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = ctx->counters.ensure(64)) != cudaSuccess || (e = cudaMemset(ctx->counters.p, 0, 64)) != cudaSuccess ||
        (e = ctx->cam.ensure(8 * sizeof(float4))) != cudaSuccess) {
        set(cudaGetErrorString(e));
        return SR_ERR_CUDA;
    }
    for (auto& ev : ctx->ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) { set(cudaGetErrorString(e)); return SR_ERR_CUDA; }
    ctx->bb = make_bb();
    if (fast_init(ctx->fast, prop) != cudaSuccess) { set("fast path init failed"); return SR_ERR_CUDA; }
    *out = ctx.release();
    return SR_OK;
}

void sr_destroy(sr_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& ev : ctx->ev) if (ev) cudaEventDestroy(ev);
    AsyncOutput& ao = ctx->async;
    if (ao.copy) {
        cudaStreamSynchronize(ao.copy);
        cudaStreamDestroy(ao.copy);
    }
    for (int b = 0; b < 2; ++b) {
        if (ao.rendered[b]) cudaEventDestroy(ao.rendered[b]);
        if (ao.copied[b]) cudaEventDestroy(ao.copied[b]);
    }
    fast_release(ctx->fast);
    ctx->scenes.clear();
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
}

const char* sr_last_error(const sr_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

sr_status sr_adapter_name(const sr_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || !len) return SR_ERR_INVALID_ARGUMENT;
    std::strncpy(buf, ctx->name.c_str(), len - 1);
    buf[len - 1] = 0;
    return SR_OK;
}

sr_status sr_set_stream(sr_ctx* ctx, void* s) {
    if (!ctx) return SR_ERR_INVALID_ARGUMENT;
    ctx->stream = s ? (cudaStream_t)s : ctx->own;
    return SR_OK;
}

}  // extern "C"

namespace {
// The device error flags a batch left in its counters (counters[1]), as a status.
sr_status batch_errors(sr_ctx* ctx, uint32_t flags) {
    if (flags & ERR_TRAVERSAL_LIMIT) return fail(ctx, SR_ERR_TRAVERSAL_LIMIT, "a ray exceeded the traversal visit limit");
    if (flags & ERR_SHADOW_MISMATCH) return fail(ctx, SR_ERR_CUDA, "internal error: shadow state mismatch");
    if (flags) return fail(ctx, SR_ERR_BAD_SCENE, "device reported a bad index");
    return SR_OK;
}

// Waits for the asynchronous batch that used framebuffer b (if any) and reports its errors.
sr_status settle_async(sr_ctx* ctx, int b) {
    AsyncOutput& ao = ctx->async;
    if (!ao.pending[b]) return SR_OK;
    CK(cudaEventSynchronize(ao.copied[b]), "async readback");
    ao.pending[b] = false;
    return batch_errors(ctx, ao.flags.as<uint32_t>()[16 * b + 1]);
}
}  // namespace

extern "C" {

sr_status sr_synchronize(sr_ctx* ctx) {
    if (!ctx) return SR_ERR_INVALID_ARGUMENT;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    sr_status first = SR_OK;
    for (int k = 0; k < 2; ++k) {  // oldest first
        const sr_status r = settle_async(ctx, (ctx->async.next + k) & 1);
        if (first == SR_OK) first = r;
    }
    return first;
}

sr_status sr_upload_scene(sr_ctx* ctx, uint32_t idx, const SrSceneDesc* d) {
    if (!ctx || !d) return SR_ERR_INVALID_ARGUMENT;
    if (idx > 4096) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "scene index too large");
    uint32_t depth = 0;
    char why[256] = {0};
    if (sr_scene_validate(d, &depth, why, sizeof(why)) != SR_OK)
        return fail(ctx, SR_ERR_BAD_SCENE, std::string("invalid scene: ") + why);
    CK(cudaSetDevice(ctx->device), "set device");
    if (ctx->scenes.size() <= idx) ctx->scenes.resize(idx + 1);
    auto slot = std::make_unique<SceneSlot>();
    SceneSlot& s = *slot;
    auto up = [&](DevBuf& b, const void* src, size_t bytes, const char* what) -> cudaError_t {
        cudaError_t e = b.ensure(std::max<size_t>(bytes, 16));
        if (e != cudaSuccess || !bytes) return e;
        return cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice);
        (void)what;
    };
    CK(up(s.nodes, d->nodes, (size_t)d->num_nodes * sizeof(SrGpuNode), "nodes"), "upload nodes");
    CK(up(s.geoms, d->geoms, (size_t)d->num_prims * sizeof(SrGpuGeom), "geoms"), "upload geoms");
    CK(up(s.attrs, d->attrs, (size_t)d->num_prims * sizeof(SrGpuAttr), "attrs"), "upload attrs");
    CK(up(s.mats, d->materials, (size_t)d->num_materials * sizeof(SrGpuMaterial), "materials"), "upload materials");
    CK(up(s.stars, d->stars, (size_t)d->num_star_vec4 * 16, "stars"), "upload stars");
    if (d->leaf_to_orig) {
        CK(up(s.l2o, d->leaf_to_orig, (size_t)d->num_prims * 4, "order"), "upload order");
        s.has_l2o = true;
    }
    s.num_nodes = d->num_nodes;
    s.num_prims = d->num_prims;
    s.empty_tree = d->num_nodes && SR_NODE_IS_NOTHING(&d->nodes[0]);
    s.num_mats = d->num_materials;
    s.num_stars = d->num_stars;
    s.num_star_vec4 = d->num_star_vec4;
    s.depth = depth;
    for (int k = 0; k < 4; ++k) {
        s.light_pos[k] = d->light_pos[k];
        s.anchor[k] = d->anchor ? d->anchor[k] : 0.0;
    }
    s.fast.layout = ctx->layout_of(idx);
    CK(fast_build(ctx->fast, s.fast, s.nodes.as<SrGpuNode>(), s.num_nodes, depth, s.num_prims, max_leaf_of(d),
                  ctx->stream),
       "build node layout");
    s.tuning = fast_default_tuning(ctx->fast);
    CK(cudaStreamSynchronize(ctx->stream), "upload sync");
    s.present = true;
    ctx->scenes[idx] = std::move(slot);
    return SR_OK;
}

sr_status sr_update_scene(sr_ctx* ctx, uint32_t idx, const SrSceneDesc* d, const SrRange* nr, uint32_t n_nr,
                          const SrRange* pr, uint32_t n_pr) {
    if (!ctx || !d) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return sr_upload_scene(ctx, idx, d);
    SceneSlot& s = *ctx->scenes[idx];
    bool fits = (size_t)d->num_nodes * sizeof(SrGpuNode) <= s.nodes.bytes &&
                (size_t)d->num_prims * sizeof(SrGpuGeom) <= s.geoms.bytes &&
                (size_t)d->num_prims * sizeof(SrGpuAttr) <= s.attrs.bytes && (size_t)d->num_star_vec4 * 16 <= s.stars.bytes &&
                d->num_materials == s.num_mats && (!d->leaf_to_orig || s.has_l2o);
    for (uint32_t i = 0; i < n_nr && fits; ++i) fits = nr[i].start <= nr[i].end && nr[i].end <= d->num_nodes;
    for (uint32_t i = 0; i < n_pr && fits; ++i) fits = pr[i].start <= pr[i].end && pr[i].end <= d->num_prims;
    if (!fits) return sr_upload_scene(ctx, idx, d);  // gpu.rs:730: upload afresh
    s.arena.reset();  // patched from the host: no longer a device scene cache's arena
    uint32_t depth = 0;
    char why[256] = {0};
    if (sr_scene_validate(d, &depth, why, sizeof(why)) != SR_OK)
        return fail(ctx, SR_ERR_BAD_SCENE, std::string("invalid scene: ") + why);
    CK(cudaSetDevice(ctx->device), "set device");
    for (uint32_t i = 0; i < n_nr; ++i) {  // write_ranges (gpu.rs:325-330)
        size_t a = nr[i].start, b = nr[i].end;
        if (b > a) CK(cudaMemcpyAsync(s.nodes.as<SrGpuNode>() + a, d->nodes + a, (b - a) * sizeof(SrGpuNode), cudaMemcpyHostToDevice, ctx->stream), "patch nodes");
    }
    for (uint32_t i = 0; i < n_pr; ++i) {
        size_t a = pr[i].start, b = pr[i].end;
        if (b <= a) continue;
        CK(cudaMemcpyAsync(s.geoms.as<SrGpuGeom>() + a, d->geoms + a, (b - a) * sizeof(SrGpuGeom), cudaMemcpyHostToDevice, ctx->stream), "patch geoms");
        CK(cudaMemcpyAsync(s.attrs.as<SrGpuAttr>() + a, d->attrs + a, (b - a) * sizeof(SrGpuAttr), cudaMemcpyHostToDevice, ctx->stream), "patch attrs");
        if (d->leaf_to_orig)
            CK(cudaMemcpyAsync(s.l2o.as<uint32_t>() + a, d->leaf_to_orig + a, (b - a) * 4, cudaMemcpyHostToDevice, ctx->stream), "patch order");
    }
    if (d->num_star_vec4)
        CK(cudaMemcpyAsync(s.stars.p, d->stars, (size_t)d->num_star_vec4 * 16, cudaMemcpyHostToDevice, ctx->stream), "patch stars");
    s.num_nodes = d->num_nodes;
    s.num_prims = d->num_prims;
    s.empty_tree = d->num_nodes && SR_NODE_IS_NOTHING(&d->nodes[0]);
    s.num_stars = d->num_stars;
    s.num_star_vec4 = d->num_star_vec4;
    s.depth = depth;
    CK(fast_build(ctx->fast, s.fast, s.nodes.as<SrGpuNode>(), s.num_nodes, depth, s.num_prims, max_leaf_of(d),
                  ctx->stream),
       "rebuild node layout");
    CK(cudaStreamSynchronize(ctx->stream), "update sync");
    return SR_OK;
}

// The slot a build fills: the index's previous scene, whose device buffers are reused when they
// are large enough (a scene rebuilt every frame allocates nothing once warm), else a new one. The
// index holds no scene until the build succeeds.
static std::unique_ptr<SceneSlot> take_slot(sr_ctx* ctx, uint32_t idx) {
    if (idx < ctx->scenes.size() && ctx->scenes[idx]) {
        cudaStreamSynchronize(ctx->stream);  // frames queued on the old scene finish first
        std::unique_ptr<SceneSlot> s = std::move(ctx->scenes[idx]);
        s->present = false;
        s->arena.reset();  // its arrays stop being a scene cache's arena
        return s;
    }
    return std::make_unique<SceneSlot>();
}

// The tree, leaf order and node layout of a scene whose simplices (build order) are on the device.
static sr_status finish_build(sr_ctx* ctx, SceneSlot& s, const float4* box, const SrGpuGeom* gin, const SrGpuAttr* ain,
                              uint32_t n, cudaStream_t st) {
    CK(s.nodes.ensure((size_t)2 * n * sizeof(SrGpuNode)), "alloc nodes");
    CK(s.l2o.ensure((size_t)n * 4), "alloc order");
    GpuBuildInfo info{};
    CK(gpu_bvh_build(box, n, s.nodes.as<SrGpuNode>(), s.l2o.as<uint32_t>(), &info, st), "build tree");
    if (info.unsupported)
        return fail(ctx, SR_ERR_UNSUPPORTED,
                    "a split left one side empty: the reference selects by median there; build this scene on the host");
    CK(s.geoms.ensure((size_t)n * sizeof(SrGpuGeom)), "alloc geoms");
    CK(s.attrs.ensure((size_t)n * sizeof(SrGpuAttr)), "alloc attrs");
    CK(gpu_gather_records(s.l2o.as<uint32_t>(), n, gin, ain, s.geoms.as<SrGpuGeom>(), s.attrs.as<SrGpuAttr>(), st),
       "leaf order");
    CK(cudaStreamSynchronize(st), "build sync");
    s.num_nodes = info.num_nodes;
    s.depth = info.depth;
    s.has_l2o = true;
    s.empty_tree = false;
    s.rindler_crossed = false;
    s.num_prims = n;
    CK(fast_build(ctx->fast, s.fast, s.nodes.as<SrGpuNode>(), s.num_nodes, s.depth, n, info.max_leaf, st),
       "build node layout");
    return SR_OK;
}

// Materials, stars, light and anchor of a built scene; the slot goes live at `idx`.
}  // extern "C"

namespace sre {
sr_status upload_scene_rest(sr_ctx* ctx, SceneSlot& s, const SrBuildDesc* d) {
    auto up = [&](DevBuf& b, const void* src, size_t bytes) -> cudaError_t {
        cudaError_t e = b.ensure(std::max<size_t>(bytes, 16));
        if (e != cudaSuccess || !bytes) return e;
        return cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice);
    };
    CK(up(s.mats, d->materials, (size_t)d->num_materials * sizeof(SrGpuMaterial)), "upload materials");
    CK(up(s.stars, d->stars, (size_t)d->num_star_vec4 * 16), "upload stars");
    s.num_mats = d->num_materials;
    s.num_stars = d->num_stars;
    s.num_star_vec4 = d->num_star_vec4;
    for (int k = 0; k < 4; ++k) {
        s.light_pos[k] = d->light_pos[k];
        s.anchor[k] = d->anchor ? d->anchor[k] : 0.0;
    }
    return SR_OK;
}
}  // namespace sre

extern "C" {

static sr_status finish_scene(sr_ctx* ctx, uint32_t idx, std::unique_ptr<SceneSlot> slot, const SrBuildDesc* d) {
    SceneSlot& s = *slot;
    sr_status r = upload_scene_rest(ctx, s, d);
    if (r != SR_OK) return r;
    s.tuning = fast_default_tuning(ctx->fast);
    CK(cudaStreamSynchronize(ctx->stream), "build sync");
    s.present = true;
    if (ctx->scenes.size() <= idx) ctx->scenes.resize(idx + 1);
    ctx->scenes[idx] = std::move(slot);
    return SR_OK;
}

// Materials and star segments checked as sr_upload_scene checks them (no tree yet).
}  // extern "C"

sr_status sre::check_build_desc(sr_ctx* ctx, const SrBuildDesc* d, const SrGpuAttr* host_attrs, uint32_t n) {
    SrSceneDesc v{};
    v.num_prims = host_attrs ? n : 0;
    v.attrs = host_attrs;
    v.geoms = host_attrs ? d->geoms : nullptr;
    v.materials = d->materials;
    v.num_materials = d->num_materials;
    v.num_stars = d->num_stars;
    v.stars = d->stars;
    v.num_star_vec4 = d->num_star_vec4;
    uint32_t unused_depth = 0;
    char why[256] = {0};
    if (sr_scene_validate(&v, &unused_depth, why, sizeof(why)) != SR_OK)
        return fail(ctx, SR_ERR_BAD_SCENE, std::string("invalid scene: ") + why);
    return SR_OK;
}

extern "C" {

sr_status sr_build_scene(sr_ctx* ctx, uint32_t idx, const SrBuildDesc* d) {
    if (!ctx || !d) return SR_ERR_INVALID_ARGUMENT;
    if (idx > 4096) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "scene index too large");
    const uint32_t n = d->num_prims;
    if (n == 0 || !d->boxes || !d->geoms || !d->attrs) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "no simplices to build");
    sr_status r = check_build_desc(ctx, d, d->attrs, n);
    if (r != SR_OK) return r;
    CK(cudaSetDevice(ctx->device), "set device");
    auto slot = take_slot(ctx, idx);
    cudaStream_t st = ctx->stream;
    {
        DevBuf box, gin, ain;
        CK(box.ensure((size_t)n * 32), "alloc boxes");
        CK(gin.ensure((size_t)n * sizeof(SrGpuGeom)), "alloc geoms");
        CK(ain.ensure((size_t)n * sizeof(SrGpuAttr)), "alloc attrs");
        CK(cudaMemcpyAsync(box.p, d->boxes, (size_t)n * 32, cudaMemcpyHostToDevice, st), "upload boxes");
        CK(cudaMemcpyAsync(gin.p, d->geoms, (size_t)n * sizeof(SrGpuGeom), cudaMemcpyHostToDevice, st), "upload geoms");
        CK(cudaMemcpyAsync(ain.p, d->attrs, (size_t)n * sizeof(SrGpuAttr), cudaMemcpyHostToDevice, st), "upload attrs");
        slot->fast.layout = ctx->layout_of(idx);
        r = finish_build(ctx, *slot, box.as<float4>(), gin.as<SrGpuGeom>(), ain.as<SrGpuAttr>(), n, st);
        if (r != SR_OK) return r;
    }
    return finish_scene(ctx, idx, std::move(slot), d);
}

sr_status sr_build_scene_tubes(sr_ctx* ctx, uint32_t idx, const SrTube* tubes, uint32_t num_tubes, const SrBuildDesc* d) {
    if (!ctx || !d || (!tubes && num_tubes)) return SR_ERR_INVALID_ARGUMENT;
    if (idx > 4096) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "scene index too large");
    for (uint32_t b = 0; b < num_tubes; ++b) {
        const SrTube& t = tubes[b];
        if ((t.num_vertices && !t.vertices) || (t.num_triangles && !t.triangles) || (t.num_samples && !t.samples))
            return fail(ctx, SR_ERR_INVALID_ARGUMENT, "tube " + std::to_string(b) + ": null array");
        if (t.material >= d->num_materials)
            return fail(ctx, SR_ERR_BAD_SCENE, "tube " + std::to_string(b) + ": material id out of range");
        for (uint32_t i = 0; i < t.num_triangles; ++i)
            for (int k = 0; k < 3; ++k)
                if (t.triangles[i].idx[k] >= t.num_vertices)
                    return fail(ctx, SR_ERR_BAD_SCENE, "tube " + std::to_string(b) + ": vertex index out of range");
        if ((uint64_t)t.num_samples * t.num_vertices > 0xFFFFFFFFull || (uint64_t)t.num_samples * t.num_triangles > 0x3FFFFFFFull)
            return fail(ctx, SR_ERR_INVALID_ARGUMENT, "tube " + std::to_string(b) + ": too many samples");
    }
    sr_status r = check_build_desc(ctx, d, nullptr, 0);
    if (r != SR_OK) return r;
    CK(cudaSetDevice(ctx->device), "set device");
    auto slot = take_slot(ctx, idx);
    cudaStream_t st = ctx->stream;
    ExtrudeOut ex{};
    cudaError_t e = gpu_extrude(tubes, num_tubes, &ex, st);
    struct Free {
        ExtrudeOut* x;
        cudaStream_t st;
        ~Free() {
            if (x->geoms) cudaFreeAsync(x->geoms, st);
            if (x->attrs) cudaFreeAsync(x->attrs, st);
            if (x->boxes) cudaFreeAsync(x->boxes, st);
        }
    } free_ex{&ex, st};
    CK(e, "extrude");
    if (ex.num_prims == 0) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "the tubes hold no simplices");
    slot->fast.layout = ctx->layout_of(idx);
    r = finish_build(ctx, *slot, ex.boxes, ex.geoms, ex.attrs, ex.num_prims, st);
    if (r != SR_OK) return r;
    slot->rindler_crossed = ex.rindler_bad != 0;
    return finish_scene(ctx, idx, std::move(slot), d);
}

sr_status sr_scene_records(sr_ctx* ctx, uint32_t idx, SrGpuGeom* geoms, SrGpuAttr* attrs, uint32_t cap) {
    if (!ctx) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "no scene at this index");
    SceneSlot& s = *ctx->scenes[idx];
    if (cap < s.num_prims) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "record buffer too small");
    if (geoms) CK(cudaMemcpy(geoms, s.geoms.p, (size_t)s.num_prims * sizeof(SrGpuGeom), cudaMemcpyDeviceToHost), "read geoms");
    if (attrs) CK(cudaMemcpy(attrs, s.attrs.p, (size_t)s.num_prims * sizeof(SrGpuAttr), cudaMemcpyDeviceToHost), "read attrs");
    return SR_OK;
}

sr_status sr_scene_tree(sr_ctx* ctx, uint32_t idx, SrGpuNode* nodes, uint32_t nodes_cap, uint32_t* order,
                        uint32_t order_cap, uint32_t* num_nodes) {
    if (!ctx || !num_nodes) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "no scene at this index");
    SceneSlot& s = *ctx->scenes[idx];
    *num_nodes = s.num_nodes;
    if (nodes) {
        if (nodes_cap < s.num_nodes) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "node buffer too small");
        CK(cudaMemcpy(nodes, s.nodes.p, (size_t)s.num_nodes * sizeof(SrGpuNode), cudaMemcpyDeviceToHost), "read nodes");
    }
    if (order) {
        if (order_cap < s.num_prims) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "order buffer too small");
        if (s.has_l2o) CK(cudaMemcpy(order, s.l2o.p, (size_t)s.num_prims * 4, cudaMemcpyDeviceToHost), "read order");
        else for (uint32_t i = 0; i < s.num_prims; ++i) order[i] = i;
    }
    return SR_OK;
}

sr_status sr_scene_stats(const sr_ctx* ctx, uint32_t idx, SrSceneStats* o) {
    if (!ctx || !o || idx >= ctx->scenes.size() || !ctx->scenes[idx]) return SR_ERR_INVALID_ARGUMENT;
    const SceneSlot& s = *ctx->scenes[idx];
    std::memset(o, 0, sizeof(*o));
    o->num_nodes = s.num_nodes;
    o->num_prims = s.num_prims;
    o->num_stars = s.num_stars;
    o->bvh_depth = s.depth;
    o->device_bytes = s.nodes.bytes + s.geoms.bytes + s.attrs.bytes + s.mats.bytes + s.stars.bytes + s.l2o.bytes + s.fast.bytes();
    o->fast_nodes = s.fast.num_wide;
    o->rindler_crossed = s.rindler_crossed ? 1u : 0u;
    o->box_copies = s.fast.num_wide ? s.fast.copies : 0u;
    return SR_OK;
}

sr_status sr_set_layout(sr_ctx* ctx, uint32_t idx, uint32_t layout) {
    if (!ctx || layout > SR_LAYOUT_COMPACT || idx > 4096) return SR_ERR_INVALID_ARGUMENT;
    if (ctx->layouts.size() <= idx) ctx->layouts.resize(idx + 1, SR_LAYOUT_AUTO);
    ctx->layouts[idx] = layout;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present) return SR_OK;
    SceneSlot& s = *ctx->scenes[idx];
    CK(cudaSetDevice(ctx->device), "set device");
    s.fast.layout = layout;
    CK(fast_build(ctx->fast, s.fast, s.nodes.as<SrGpuNode>(), s.empty_tree ? 0u : s.num_nodes, s.depth, s.num_prims,
                  s.fast.max_leaf, ctx->stream),
       "rebuild node layout");
    return SR_OK;
}

sr_status sr_get_tuning(const sr_ctx* ctx, uint32_t idx, SrTuning* t) {
    if (!ctx || !t || idx >= ctx->scenes.size() || !ctx->scenes[idx]) return SR_ERR_INVALID_ARGUMENT;
    *t = ctx->scenes[idx]->tuning;
    return SR_OK;
}

sr_status sr_set_tuning(sr_ctx* ctx, uint32_t idx, const SrTuning* t) {
    if (!ctx || !t || idx >= ctx->scenes.size() || !ctx->scenes[idx]) return SR_ERR_INVALID_ARGUMENT;
    if (!fast_tuning_valid(ctx->fast, *t)) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "tuning outside the supported set");
    ctx->scenes[idx]->tuning = *t;
    return SR_OK;
}

sr_status sr_render_ex(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, const SrRenderOpts* opts, const SrOutputs* out,
                       SrTimings* timings) {
    if (!ctx || !u || !out || !out->rgb) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "scene " + std::to_string(idx) + " is not uploaded");
    if (u->size[0] == 0 || u->size[1] == 0 || (uint64_t)u->size[0] * u->size[1] > (1ull << 28))
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "frame size must be non-zero and at most 2^28 pixels");
    if (u->mode > 3 || u->shadow_mode > 2 || u->slice_mode > 3 || u->num_flashes > SR_MAX_FLASHES || u->num_haze > SR_MAX_HAZE_ORIGINS)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "uniform block out of range");
    SceneSlot& s = *ctx->scenes[idx];
    const uint32_t path = opts ? opts->path : SR_PATH_FAST;
    const uint32_t flags = opts ? opts->flags : 0u;
    const bool count = (flags & SR_FLAG_COUNT_WORK) != 0;
    const bool dev_out = (flags & SR_FLAG_DEVICE_OUTPUT) != 0 && !count;
    const bool timing = (flags & SR_FLAG_TIMING) != 0;
    if (path != SR_PATH_PLAIN && path != SR_PATH_FAST) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "unknown path");
    if (count && (flags & SR_FLAG_DEVICE_OUTPUT)) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "work counting returns host outputs");
    CK(cudaSetDevice(ctx->device), "set device");
    sr_status st = ensure_frame(ctx, u->size[0], u->size[1]);
    if (st != SR_OK) return st;
    Frame& fr = ctx->frame;
    const size_t npx = (size_t)u->size[0] * u->size[1];
    FrameDev f{};
    f.hdr = fr.hdr.as<float4>();
    f.width = u->size[0];
    f.height = u->size[1];
    f.counters = ctx->counters.as<uint32_t>();
    if (dev_out) {
        f.rgb = out->rgb;
        f.hit_id = out->hit_id;
        f.lambda = out->lambda;
        f.tau = out->tau;
    } else {
        f.rgb = fr.rgb.as<uint32_t>();
        if (out->hit_id) { CK(fr.hit.ensure(npx * 4), "aux"); f.hit_id = fr.hit.as<uint32_t>(); }
        if (out->lambda) { CK(fr.lam.ensure(npx * 4), "aux"); f.lambda = fr.lam.as<float>(); }
        if (out->tau) { CK(fr.tau.ensure(npx * 4), "aux"); f.tau = fr.tau.as<float>(); }
    }
    cudaStream_t sm = ctx->stream;
    cudaEvent_t* ev = ctx->ev;
    auto t_host0 = std::chrono::steady_clock::now();
    SceneDev sd = scene_dev(ctx, s);
    const void* hdr_src = fr.hdr.p;
    if (path == SR_PATH_PLAIN || !s.fast.usable) {
        if (timing) CK(cudaEventRecord(ev[0], sm), "event");
        CK(cudaMemsetAsync(ctx->counters.p, 0, count ? 64 : 16, sm), "counters");
        const float4* cam_dev = nullptr;
        if (opts && opts->cam64) {
            CK(launch_camera_f64(*opts->cam64, s.anchor, *u, ctx->cam.as<float4>(), sm), "camera kernel");
            cam_dev = ctx->cam.as<float4>();
        }
        if (timing) CK(cudaEventRecord(ev[1], sm), "event");
        CK(launch_render_plain(sd, *u, cam_dev, f, ctx->bb, sm), "plain render");
        if (timing) for (int k = 2; k <= 4; ++k) CK(cudaEventRecord(ev[k], sm), "event");
        CK(launch_bloom(f, fr.pyr, ctx->tables.as<uint32_t>(), sm), "bloom");
        if (timing) CK(cudaEventRecord(ev[5], sm), "event");
    } else {
        // The fast path renders a single frame as a batch of one observer.
        BatchRequest br{};
        br.n = 1;
        br.u = u;
        br.cam64 = opts ? opts->cam64 : nullptr;
        br.rgb = f.rgb;
        br.hit_id = f.hit_id;
        br.lambda = f.lambda;
        br.tau = f.tau;
        br.count_work = count;
        br.use_graph = !timing && !count;
        br.star_brute = (flags & SR_FLAG_STAR_BRUTE) != 0;
        br.ev = timing ? ev + 1 : nullptr;
        if (timing) CK(cudaEventRecord(ev[0], sm), "event");
        CK(fast_render_batch(ctx->fast, s.fast, s.tuning, sd, s.anchor, ctx->bb, ctx->counters.as<uint32_t>(), br, sm),
           "fast render");
        // Events [1]..[5]: camera, trace, shading (+ shadow rays and stars), the same point, bloom.
        hdr_src = fast_batch_hdr(ctx->fast, 0);
    }
    if (out->hdr) CK(cudaMemcpyAsync(out->hdr, hdr_src, npx * 16, dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, sm), "hdr copy");
    if (dev_out && !timings) return SR_OK;
    auto t_host1 = std::chrono::steady_clock::now();
    if (!dev_out) {
        CK(cudaMemcpyAsync(out->rgb, f.rgb, npx * 4, cudaMemcpyDeviceToHost, sm), "readback");
        if (out->hit_id) CK(cudaMemcpyAsync(out->hit_id, f.hit_id, npx * 4, cudaMemcpyDeviceToHost, sm), "readback");
        if (out->lambda) CK(cudaMemcpyAsync(out->lambda, f.lambda, npx * 4, cudaMemcpyDeviceToHost, sm), "readback");
        if (out->tau) CK(cudaMemcpyAsync(out->tau, f.tau, npx * 4, cudaMemcpyDeviceToHost, sm), "readback");
    }
    uint32_t counters[16] = {0};
    CK(cudaMemcpyAsync(counters, ctx->counters.p, 64, cudaMemcpyDeviceToHost, sm), "counters");
    CK(cudaStreamSynchronize(sm), "render sync");
    auto t_host2 = std::chrono::steady_clock::now();
    if (timings) {
        std::memset(timings, 0, sizeof(*timings));
        timings->submit_ms = std::chrono::duration<float, std::milli>(t_host1 - t_host0).count();
        timings->wait_ms = std::chrono::duration<float, std::milli>(t_host2 - t_host1).count();
        timings->shadow_rays = counters[0];
        if (count && path == SR_PATH_FAST) {
            uint64_t w[6];
            std::memcpy(w, counters + 4, sizeof(w));
            timings->nodes_visited = w[0];
            timings->leaves_visited = w[1];
            timings->tets_tested = w[2];
            timings->shadow_nodes_visited = w[3];
            timings->shadow_leaves_visited = w[4];
            timings->shadow_tets_tested = w[5];
        }
        if (timing) {
            cudaEventElapsedTime(&timings->kernel_ms, ev[0], ev[5]);
            cudaEventElapsedTime(&timings->camera_ms, ev[0], ev[1]);
            cudaEventElapsedTime(&timings->trace_ms, ev[1], ev[2]);
            cudaEventElapsedTime(&timings->shade_ms, ev[2], ev[3]);
            cudaEventElapsedTime(&timings->stars_ms, ev[3], ev[4]);
            cudaEventElapsedTime(&timings->bloom_ms, ev[4], ev[5]);
        }
    }
    if (counters[1] & ERR_TRAVERSAL_LIMIT) return fail(ctx, SR_ERR_TRAVERSAL_LIMIT, "a ray exceeded the traversal visit limit");
    if (counters[1] & ERR_SHADOW_MISMATCH) return fail(ctx, SR_ERR_CUDA, "internal error: shadow state mismatch");
    if (counters[1]) return fail(ctx, SR_ERR_BAD_SCENE, "device reported a bad index (flags " + std::to_string(counters[1]) + ")");
    return SR_OK;
}

sr_status sr_render(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, uint32_t* fb, uint64_t fb_len, SrTimings* t) {
    if (!ctx || !u || !fb) return SR_ERR_INVALID_ARGUMENT;
    if (fb_len != (uint64_t)u->size[0] * u->size[1])
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "framebuffer size mismatch");  // gpu.rs:808
    SrOutputs o{};
    o.rgb = fb;
    return sr_render_ex(ctx, idx, u, nullptr, &o, t);
}

sr_status sr_trace_rays(sr_ctx* ctx, uint32_t idx, const SrRay* rays, uint32_t n, SrRayHit* hits) {
    if (!ctx || (n && (!rays || !hits))) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "scene " + std::to_string(idx) + " is not uploaded");
    if (n == 0) return SR_OK;
    CK(cudaSetDevice(ctx->device), "set device");
    SceneSlot& s = *ctx->scenes[idx];
    DevBuf din, dout;
    CK(din.ensure((size_t)n * sizeof(SrRay)), "ray buffer");
    CK(dout.ensure((size_t)n * sizeof(SrRayHit)), "hit buffer");
    cudaStream_t sm = ctx->stream;
    CK(cudaMemcpyAsync(din.p, rays, (size_t)n * sizeof(SrRay), cudaMemcpyHostToDevice, sm), "rays in");
    CK(cudaMemsetAsync(ctx->counters.p, 0, 16, sm), "clear counters");
    CK(launch_trace_rays(scene_dev(ctx, s), s.anchor, din.as<SrRay>(), n, dout.as<SrRayHit>(), ctx->counters.as<uint32_t>(),
                         sm),
       "ray kernel");
    CK(cudaMemcpyAsync(hits, dout.p, (size_t)n * sizeof(SrRayHit), cudaMemcpyDeviceToHost, sm), "hits out");
    uint32_t counters[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(counters, ctx->counters.p, 16, cudaMemcpyDeviceToHost, sm), "counters");
    CK(cudaStreamSynchronize(sm), "ray sync");
    if (counters[1] & ERR_TRAVERSAL_LIMIT) return fail(ctx, SR_ERR_TRAVERSAL_LIMIT, "a ray exceeded the traversal visit limit");
    if (counters[1]) return fail(ctx, SR_ERR_BAD_SCENE, "device reported a bad index (flags " + std::to_string(counters[1]) + ")");
    return SR_OK;
}

sr_status sr_render_batch(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, const SrCameraF64* cam64, uint32_t n,
                          uint32_t* rgb_out, uint64_t rgb_len, uint32_t flags, SrTimings* timings) {
    if (!ctx || (!u && n) || (!rgb_out && n)) return SR_ERR_INVALID_ARGUMENT;
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) total += (uint64_t)u[i].size[0] * u[i].size[1];
    if (total != rgb_len) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "rgb_len must equal the sum of the observers' pixels");
    if (n == 0) return SR_OK;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "scene " + std::to_string(idx) + " is not uploaded");
    for (uint32_t i = 0; i < n; ++i)
        if (u[i].size[0] == 0 || u[i].size[1] == 0 || u[i].mode > 3 || u[i].shadow_mode > 2 || u[i].slice_mode > 3 ||
            u[i].num_flashes > SR_MAX_FLASHES || u[i].num_haze > SR_MAX_HAZE_ORIGINS)
            return fail(ctx, SR_ERR_INVALID_ARGUMENT, "uniform block of observer " + std::to_string(i) + " out of range");
    if (total > (1ull << 30)) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "batch larger than 2^30 pixels");
    SceneSlot& s = *ctx->scenes[idx];
    const bool dev_out = (flags & SR_FLAG_DEVICE_OUTPUT) != 0;
    const bool async_out = (flags & SR_FLAG_ASYNC_OUTPUT) != 0;
    if (async_out && (dev_out || timings))
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "SR_FLAG_ASYNC_OUTPUT takes a host framebuffer and no timings");
    CK(cudaSetDevice(ctx->device), "set device");
    cudaStream_t sm = ctx->stream;
    cudaEvent_t* ev = ctx->ev;
    if (async_out && s.fast.usable) {
        // The batch renders into framebuffer b once the readback of the batch before that used it
        // has finished; its readback then runs on the copy stream while the next batch renders.
        AsyncOutput& ao = ctx->async;
        if (!ao.copy) {
            CK(cudaStreamCreateWithFlags(&ao.copy, cudaStreamNonBlocking), "copy stream");
            for (int b = 0; b < 2; ++b) {
                CK(cudaEventCreateWithFlags(&ao.rendered[b], cudaEventDisableTiming), "event");
                CK(cudaEventCreateWithFlags(&ao.copied[b], cudaEventDisableTiming), "event");
            }
            CK(ao.flags.ensure(2 * 16 * sizeof(uint32_t)), "pinned flags");
        }
        const int b = ao.next;
        sr_status r = settle_async(ctx, b);
        if (r != SR_OK) return r;
        CK(ao.rgb[b].ensure(total * 4), "framebuffer");
        BatchRequest br{};
        br.n = n;
        br.u = u;
        br.cam64 = cam64;
        br.rgb = ao.rgb[b].as<uint32_t>();
        br.use_graph = true;
        br.star_brute = (flags & SR_FLAG_STAR_BRUTE) != 0;
        SceneDev sd = scene_dev(ctx, s);
        CK(fast_render_batch(ctx->fast, s.fast, s.tuning, sd, s.anchor, ctx->bb, ctx->counters.as<uint32_t>(), br, sm),
           "batch render");
        CK(cudaMemcpyAsync(ao.flags.as<uint32_t>() + 16 * b, ctx->counters.p, 64, cudaMemcpyDeviceToHost, sm), "flags");
        CK(cudaEventRecord(ao.rendered[b], sm), "event");
        CK(cudaStreamWaitEvent(ao.copy, ao.rendered[b], 0), "event");
        CK(cudaMemcpyAsync(rgb_out, ao.rgb[b].p, total * 4, cudaMemcpyDeviceToHost, ao.copy), "batch readback");
        CK(cudaEventRecord(ao.copied[b], ao.copy), "event");
        ao.pending[b] = true;
        ao.next = 1 - b;
        return SR_OK;
    }
    if (!s.fast.usable) {  // trees the fast path cannot take render one by one on the plain path
        DevBuf staging;
        uint32_t* dst = rgb_out;
        if (!dev_out) {
            CK(staging.ensure(total * 4), "batch staging");
            dst = staging.as<uint32_t>();
        }
        if (timings) CK(cudaEventRecord(ev[6], sm), "event");
        uint64_t off = 0;
        for (uint32_t i = 0; i < n; ++i) {
            SrRenderOpts o{SR_PATH_PLAIN, SR_FLAG_DEVICE_OUTPUT, cam64 ? cam64 + i : nullptr};
            SrOutputs out{};
            out.rgb = dst + off;
            sr_status st = sr_render_ex(ctx, idx, u + i, &o, &out, nullptr);
            if (st != SR_OK) return st;
            off += (uint64_t)u[i].size[0] * u[i].size[1];
        }
        if (timings) CK(cudaEventRecord(ev[7], sm), "event");
        if (!dev_out) CK(cudaMemcpyAsync(rgb_out, dst, total * 4, cudaMemcpyDeviceToHost, sm), "batch readback");
    } else {
        BatchRequest br{};
        br.n = n;
        br.u = u;
        br.cam64 = cam64;
        br.rgb = dev_out ? rgb_out : nullptr;
        br.use_graph = true;
        br.star_brute = (flags & SR_FLAG_STAR_BRUTE) != 0;
        // Per-phase events and work counting run the sequence outside its graph.
        br.ev = (timings && (flags & SR_FLAG_TIMING)) ? ev + 1 : nullptr;
        br.count_work = timings && (flags & SR_FLAG_COUNT_WORK);
        SceneDev sd = scene_dev(ctx, s);
        if (timings) CK(cudaEventRecord(ev[6], sm), "event");
        CK(fast_render_batch(ctx->fast, s.fast, s.tuning, sd, s.anchor, ctx->bb, ctx->counters.as<uint32_t>(), br, sm),
           "batch render");
        if (timings) CK(cudaEventRecord(ev[7], sm), "event");
        if (!dev_out) CK(cudaMemcpyAsync(rgb_out, ctx->fast.rgb.p, total * 4, cudaMemcpyDeviceToHost, sm), "batch readback");
    }
    if (!dev_out || timings) {
        uint32_t counters[16] = {0};
        CK(cudaMemcpyAsync(counters, ctx->counters.p, 64, cudaMemcpyDeviceToHost, sm), "counters");
        CK(cudaStreamSynchronize(sm), "batch sync");
        if (timings) {
            std::memset(timings, 0, sizeof(*timings));
            cudaEventElapsedTime(&timings->kernel_ms, ev[6], ev[7]);
            timings->shadow_rays = counters[0];
            if (s.fast.usable && (flags & SR_FLAG_TIMING)) {
                cudaEventElapsedTime(&timings->camera_ms, ev[6], ev[1]);
                cudaEventElapsedTime(&timings->trace_ms, ev[1], ev[2]);
                cudaEventElapsedTime(&timings->shade_ms, ev[2], ev[3]);
                cudaEventElapsedTime(&timings->stars_ms, ev[3], ev[4]);
                cudaEventElapsedTime(&timings->bloom_ms, ev[4], ev[5]);
            }
            if (s.fast.usable && (flags & SR_FLAG_COUNT_WORK)) {
                uint64_t w[6];
                std::memcpy(w, counters + 4, sizeof(w));
                timings->nodes_visited = w[0];
                timings->leaves_visited = w[1];
                timings->tets_tested = w[2];
                timings->shadow_nodes_visited = w[3];
                timings->shadow_leaves_visited = w[4];
                timings->shadow_tets_tested = w[5];
            }
        }
        return batch_errors(ctx, counters[1]);
    }
    return SR_OK;
}

sr_status sr_autotune(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, uint32_t n, SrTuning* best, float* best_ms) {
    if (!ctx || !u || idx >= ctx->scenes.size() || !ctx->scenes[idx]) return SR_ERR_INVALID_ARGUMENT;
    SceneSlot& s = *ctx->scenes[idx];
    // What is tuned is the batched path, so a candidate is timed on a batch of `n` copies of the
    // observer (one launch sequence, replayed from its captured graph), after a warm-up batch.
    const uint32_t frames = std::max(1u, std::min(n, 64u));
    const size_t npx = (size_t)u->size[0] * u->size[1];
    DevBuf out;
    CK(out.ensure(npx * 4 * frames), "autotune output");
    std::vector<SrGpuUniforms> us(frames, *u);
    SrTuning keep = s.tuning;
    // The schedules worth timing: whole-warp refills of single tiles were fastest on every scene
    // measured (wider chunks or partial refills spread the rays in flight over more of the tree).
    // Per block shape and tile: the packet traversal, cooperative leaf tests, or the lean kernel
    // with the traversal stack in local memory or its first 8..16 entries in shared memory.
    const uint32_t shapes[][2] = {{128, 8}, {128, 9}, {128, 11}, {256, 4}, {256, 6}, {512, 3}, {64, 16}};
    const uint32_t tiles[][2] = {{8, 4}, {4, 8}};
    // With the stack in local memory or 12 entries in shared memory, also the top 4, 6 or 8 levels
    // of the tree staged in shared memory.
    const uint32_t stacks[][2] = {{0, 0}, {8, 0}, {10, 0}, {12, 0}, {16, 0}, {0, 4}, {0, 6}, {0, 8},
                                  {12, 4}, {12, 6}, {12, 8}};
    std::vector<SrTuning> cand{keep};
    for (auto& sh : shapes)
        for (auto& tl : tiles)
            for (uint32_t v = 0; v <= sizeof(stacks) / sizeof(stacks[0]) + 1; ++v) {
                const bool packet = v == sizeof(stacks) / sizeof(stacks[0]) + 1;
                SrTuning t = keep;
                t.block_threads = sh[0];
                t.blocks_per_sm = sh[1];
                t.tile_w = tl[0];
                t.tile_h = tl[1];
                t.chunk_tiles = 1;
                t.refill_lanes = 32;
                t.leaf_coop = v == 0 ? 1u : 0u;
                t.leaf_batch = 1;
                t.home_pct = 0;
                t.stack_smem = v == 0 || packet ? 0u : stacks[v - 1][0];
                t.top_levels = v == 0 || packet ? 0u : stacks[v - 1][1];
                t.packet = packet ? 1u : 0u;
                if (fast_tuning_valid(ctx->fast, t)) cand.push_back(t);
            }
    auto time_batch = [&](const SrTuning& t, float* ms) -> sr_status {
        s.tuning = t;
        sr_status st = sr_render_batch(ctx, idx, us.data(), nullptr, frames, out.as<uint32_t>(), npx * frames,
                                       SR_FLAG_DEVICE_OUTPUT, nullptr);  // warm-up (captures the graph)
        if (st != SR_OK) return st;
        CK(cudaEventRecord(ctx->ev[6], ctx->stream), "event");
        st = sr_render_batch(ctx, idx, us.data(), nullptr, frames, out.as<uint32_t>(), npx * frames,
                             SR_FLAG_DEVICE_OUTPUT, nullptr);
        if (st != SR_OK) return st;
        CK(cudaEventRecord(ctx->ev[7], ctx->stream), "event");
        CK(cudaEventSynchronize(ctx->ev[7]), "event sync");
        *ms = 0.0f;
        cudaEventElapsedTime(ms, ctx->ev[6], ctx->ev[7]);
        return SR_OK;
    };
    // Two sweeps, each candidate's best of the two; the current tuning (first) is kept unless a
    // candidate beats it by at least 1%, so timing noise does not move it.
    std::vector<float> ms(cand.size(), INFINITY);
    for (int sweep = 0; sweep < 2; ++sweep)
        for (size_t i = 0; i < cand.size(); ++i) {
            float m = 0.0f;
            sr_status st = time_batch(cand[i], &m);
            if (st != SR_OK) {
                s.tuning = keep;
                return st;
            }
            ms[i] = std::min(ms[i], m);
        }
    size_t win = 0;
    for (size_t i = 1; i < cand.size(); ++i)
        if (ms[i] < ms[win] && ms[i] < 0.99f * ms[0]) win = i;
    s.tuning = cand[win];
    if (best) *best = cand[win];
    if (best_ms) *best_ms = ms[win] / (float)frames;
    return SR_OK;
}

sr_status sr_adjoint(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, const SrCameraF64* cam, const float* target_hdr,
                     uint32_t level, uint32_t flags, SrAdjointResult* out) {
    if (!ctx || !u) return SR_ERR_INVALID_ARGUMENT;
    uint32_t rows = u->size[1];
    for (uint32_t k = 0; k < level && k < SR_BLOOM_LEVELS; ++k) rows = (rows + 1) / 2;
    return sr_adjoint_rows(ctx, idx, u, cam, target_hdr, level, flags, 0, rows, out);
}

sr_status sr_adjoint_rows(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, const SrCameraF64* cam,
                          const float* target_hdr, uint32_t level, uint32_t flags, uint32_t row_begin, uint32_t row_end,
                          SrAdjointResult* out) {
    if (!ctx || !u || !cam || !target_hdr || !out) return SR_ERR_INVALID_ARGUMENT;
    if (level > SR_BLOOM_LEVELS) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "loss level must be 0..6");
    uint32_t level_rows = u->size[1];
    for (uint32_t k = 0; k < level; ++k) level_rows = (level_rows + 1) / 2;
    if (row_begin >= row_end || row_end > level_rows)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "rows must be a non-empty range of the loss level's rows");
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "scene " + std::to_string(idx) + " is not uploaded");
    if (u->size[0] == 0 || u->size[1] == 0 || (uint64_t)u->size[0] * u->size[1] > (1ull << 28))
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "frame size must be non-zero and at most 2^28 pixels");
    if (u->mode != 0 || u->slice_mode != 0 || u->num_flashes != 0 || u->num_haze != 0 || u->shadow_mode > 2)
        return fail(ctx, SR_ERR_UNSUPPORTED, "the gradient covers shaded past-light-cone frames without flashes or haze");
    SceneSlot& s = *ctx->scenes[idx];
    if (!s.fast.usable) return fail(ctx, SR_ERR_UNSUPPORTED, "the gradient needs a scene the fast path takes");
    if (s.num_stars > 0 && !stars_binned_for(*u, s.num_stars))
        return fail(ctx, SR_ERR_UNSUPPORTED, "the gradient needs binned stars (field of view and pixel size of stars_binned_for)");
    CK(cudaSetDevice(ctx->device), "set device");
    const bool frozen = (flags & SR_ADJ_FROZEN) != 0;
    if (frozen && (!ctx->fast.adj_valid || ctx->fast.adj_w != u->size[0] || ctx->fast.adj_h != u->size[1] ||
                   ctx->fast.adj_geoms != scene_dev(ctx, s).geoms || ctx->fast.adj_level != level ||
                   ctx->fast.adj_r0 != row_begin || ctx->fast.adj_r1 != row_end))
        return fail(ctx, SR_ERR_INVALID_ARGUMENT,
                    "a frozen evaluation needs a gradient call on this scene, frame size, level and rows just before");
    double r[10];
    CK(fast_adjoint(ctx->fast, s.fast, s.tuning, scene_dev(ctx, s), s.anchor, ctx->bb, ctx->counters.as<uint32_t>(), *u, *cam,
                    target_hdr, level, frozen, row_begin, row_end, r, ctx->stream),
       "gradient");
    uint32_t counters[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(counters, ctx->counters.p, 16, cudaMemcpyDeviceToHost), "counters");
    if (counters[1] & ERR_TRAVERSAL_LIMIT) return fail(ctx, SR_ERR_TRAVERSAL_LIMIT, "a ray exceeded the traversal visit limit");
    if (counters[1]) return fail(ctx, SR_ERR_BAD_SCENE, "device reported a bad index (flags " + std::to_string(counters[1]) + ")");
    out->loss = r[0];
    for (int k = 0; k < 7; ++k) out->grad[k] = r[1 + k];
    out->primal_mismatch = r[8];
    out->star_terms = r[9];
    return SR_OK;
}

// ---------------------------------------------------------------------------------------------
// sr_render_noalloc: the plain path with all of its scratch in one static device array.
// ---------------------------------------------------------------------------------------------

// Layout of the array: error counters at 0 (the kernels' counters[0..3]), the six float4 rows of
// the FP64 camera at 256, the HDR image and its bloom pyramid from 512 on.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SR_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr size_t NOALLOC_COUNTERS = 0, NOALLOC_CAM = 256, NOALLOC_HDR = 512;

// Float4 entries of the HDR image and its bloom levels for a w x h frame (each level halves both
// sides, rounding up).
constexpr uint64_t noalloc_pyramid_len(uint64_t w, uint64_t h) {
    uint64_t n = 0;
    for (int k = 0; k <= SR_BLOOM_LEVELS; ++k) {
        n += w * h;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    return n;
}
// The largest pyramid of a frame within SR_NOALLOC_MAX_PIXELS is the one-row (or one-column) frame
// of all of them: its levels shrink by 2 instead of 4.
static_assert(NOALLOC_HDR + noalloc_pyramid_len(SR_NOALLOC_MAX_PIXELS, 1) * 16 <= SR_NOALLOC_SCRATCH_BYTES,
              "the no-allocation scratch holds the pyramid of every frame within the pixel limit");

// The device address of g_noalloc_scratch on the current device. In host code the array's name only
// identifies the symbol; its address comes from cudaGetSymbolAddress, looked up on every call (a
// host-side table lookup once the module is loaded), so no address outlives the context it came
// from (a cudaDeviceReset by the application between calls included).
cudaError_t noalloc_base(unsigned char** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

}  // namespace

sr_status sr_render_noalloc(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, const SrCameraF64* cam64,
                            uint32_t* rgb_dev) {
    if (!ctx || !u || !rgb_dev) return SR_ERR_INVALID_ARGUMENT;
    if (idx >= ctx->scenes.size() || !ctx->scenes[idx] || !ctx->scenes[idx]->present)
        return fail(ctx, SR_ERR_NO_SCENE, "scene " + std::to_string(idx) + " is not uploaded");
    const uint64_t npx = (uint64_t)u->size[0] * u->size[1];
    if (npx == 0) return fail(ctx, SR_ERR_INVALID_ARGUMENT, "frame size must be non-zero");
    if (npx > SR_NOALLOC_MAX_PIXELS)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT,
                    "frame of " + std::to_string(npx) + " pixels exceeds the no-allocation limit of " +
                        std::to_string(SR_NOALLOC_MAX_PIXELS) + " pixels (SR_NOALLOC_MAX_PIXELS)");
    if (u->mode > 3 || u->shadow_mode > 2 || u->slice_mode > 3 || u->num_flashes > SR_MAX_FLASHES || u->num_haze > SR_MAX_HAZE_ORIGINS)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "uniform block out of range");
    const Pyramid pyr = make_pyramid(u->size[0], u->size[1]);
    // Defensive: the static_assert above shows every frame within the pixel limit fits.
    if (NOALLOC_HDR + (size_t)pyr.off[SR_BLOOM_LEVELS + 1] * sizeof(float4) > SR_NOALLOC_SCRATCH_BYTES)
        return fail(ctx, SR_ERR_INVALID_ARGUMENT, "frame's bloom pyramid exceeds the no-allocation scratch");
    CK(cudaSetDevice(ctx->device), "set device");
    unsigned char* base = nullptr;
    CK(noalloc_base(&base), "no-allocation scratch address");
    SceneSlot& s = *ctx->scenes[idx];
    FrameDev f{};
    f.hdr = reinterpret_cast<float4*>(base + NOALLOC_HDR);
    f.rgb = rgb_dev;
    f.counters = reinterpret_cast<uint32_t*>(base + NOALLOC_COUNTERS);
    f.width = u->size[0];
    f.height = u->size[1];
    cudaStream_t sm = ctx->stream;
    // Only the counters must start at zero: the camera rows, every HDR pixel and every pyramid
    // level are written before they are read.
    CK(cudaMemsetAsync(f.counters, 0, 4 * sizeof(uint32_t), sm), "clear counters");
    const float4* cam_dev = nullptr;
    if (cam64) {
        float4* rows = reinterpret_cast<float4*>(base + NOALLOC_CAM);
        CK(launch_camera_f64(*cam64, s.anchor, *u, rows, sm), "camera kernel");
        cam_dev = rows;
    }
    CK(launch_render_plain(scene_dev(ctx, s), *u, cam_dev, f, ctx->bb, sm), "plain render");
    CK(launch_bloom(f, pyr, ctx->tables.as<uint32_t>(), sm), "bloom");
    uint32_t counters[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(counters, f.counters, sizeof(counters), cudaMemcpyDeviceToHost, sm), "counters");
    CK(cudaStreamSynchronize(sm), "render sync");
    if (counters[1] & ERR_TRAVERSAL_LIMIT) return fail(ctx, SR_ERR_TRAVERSAL_LIMIT, "a ray exceeded the traversal visit limit");
    if (counters[1]) return fail(ctx, SR_ERR_BAD_SCENE, "device reported a bad index (flags " + std::to_string(counters[1]) + ")");
    return SR_OK;
}

}  // extern "C"
