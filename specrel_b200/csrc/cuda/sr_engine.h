// Internal to the library: the context and scene slots behind the C ABI (sr_engine.cu), shared
// with the scene cache (sr_arena.cu).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../../include/specrel.h"
#include "sr_fast.h"
#include "sr_kernels.h"

namespace sre {

using namespace srk;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (n == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct ArenaCache;  // sr_arena.cu

struct SceneSlot {
    bool present = false;
    DevBuf nodes, geoms, attrs, mats, stars, l2o;
    uint32_t num_nodes = 0, num_prims = 0, num_mats = 0, num_stars = 0;
    uint64_t num_star_vec4 = 0;
    float light_pos[4] = {0, 0, 0, 0};
    double anchor[4] = {0, 0, 0, 0};
    uint32_t depth = 0;
    bool has_l2o = false;
    bool empty_tree = false;  // node 0 is BvhNode4D::NOTHING: nothing to trace
    bool rindler_crossed = false;  // built from a tube that crosses its Rindler horizon
    FastScene fast;  // the B200 node layout
    SrTuning tuning{};
    std::shared_ptr<ArenaCache> arena;  // the scene cache whose arena these arrays are, if any
};

struct Frame {
    uint32_t w = 0, h = 0;
    Pyramid pyr{};
    DevBuf hdr, rgb, hit, lam, tau;
};

// Batches with SR_FLAG_ASYNC_OUTPUT: two device framebuffers used in turn, the readbacks on a copy
// stream ordered by events, each batch's error flags in pinned memory until they are checked.
struct AsyncOutput {
    cudaStream_t copy = nullptr;
    cudaEvent_t rendered[2] = {}, copied[2] = {};
    DevBuf rgb[2];
    HostMem flags;  // 2 x 16 words: the batch's counters
    bool pending[2] = {false, false};
    int next = 0;
};

}  // namespace sre

struct sr_ctx {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::string last_error;
    std::string name;
    sre::DevBuf tables, counters, cam;
    srk::BBConst bb{};
    std::vector<std::unique_ptr<sre::SceneSlot>> scenes;
    sre::Frame frame;
    cudaEvent_t ev[8] = {};
    srk::FastCtx fast;
    sre::AsyncOutput async;
    std::vector<uint32_t> layouts;  // per scene index: SR_LAYOUT_* (default SR_LAYOUT_AUTO)
    uint32_t layout_of(uint32_t idx) const { return idx < layouts.size() ? layouts[idx] : SR_LAYOUT_AUTO; }
};

namespace sre {

inline sr_status fail(sr_ctx* c, sr_status s, const std::string& m) {
    if (c) c->last_error = m;
    return s;
}
inline sr_status cuda_fail(sr_ctx* c, cudaError_t e, const char* where) {
    return fail(c, e == cudaErrorMemoryAllocation ? SR_ERR_OUT_OF_MEMORY : SR_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(expr, where)                                \
    do {                                               \
        cudaError_t e_ = (expr);                       \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

// Materials, stars, light and anchor of `d` into slot `s` (device copies).
sr_status upload_scene_rest(sr_ctx* ctx, SceneSlot& s, const SrBuildDesc* d);
// Materials and star segments of `d` checked as sr_upload_scene checks them (and, with
// host_attrs, the material ids of n simplices).
sr_status check_build_desc(sr_ctx* ctx, const SrBuildDesc* d, const SrGpuAttr* host_attrs, uint32_t n);

}  // namespace sre
