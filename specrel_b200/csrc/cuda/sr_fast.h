// The fast path: the B200 node layout of a scene and the batched render sequence.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <vector>

#include "../../../include/specrel.h"
#include "sr_kernels.h"

namespace srk {

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { if (p) cudaFree(p); }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (!n) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    // As ensure, but a buffer that has to grow grows by a quarter more than asked, so that a scene
    // rebuilt with slowly growing arrays (an arena) does not reallocate at every rebuild.
    cudaError_t ensure_grow(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        return ensure(p ? std::max(n, bytes + bytes / 4) : n);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct HostMem {  // pinned host staging
    void* p = nullptr;
    size_t bytes = 0;
    HostMem() = default;
    HostMem(const HostMem&) = delete;
    HostMem& operator=(const HostMem&) = delete;
    ~HostMem() { if (p) cudaFreeHost(p); }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) { cudaFreeHost(p); p = nullptr; bytes = 0; }
        if (!n) return cudaSuccess;
        cudaError_t e = cudaMallocHost(&p, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// The B200 node layout of one scene (see sr_traverse.cuh).
struct FastScene {
    DevMem boxes, refs, scratch;
    // Up links for the packet traversal's ordering of equal-lambda hits (WideScene::up / leafpar).
    DevMem up, leafpar;
    uint32_t num_wide = 0;
    uint32_t depth = 0;
    uint32_t root_ref = 0;
    bool empty = true;
    bool usable = false;  // false: the scene renders on the plain path (see fast_build)
    uint32_t layout = 0;  // SR_LAYOUT_* preference for the next build
    uint32_t copies = 0;  // box copies built: 16 (one per sign octant) or 1 (compact)
    uint32_t max_leaf = 0;  // most primitives in a leaf, as the last build saw
    uint32_t top_end[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // wide nodes in the top k + 1 levels (breadth-first prefix)
    float root_min[4] = {0, 0, 0, 0}, root_max[4] = {0, 0, 0, 0};
    size_t bytes() const { return boxes.bytes + refs.bytes + up.bytes + leafpar.bytes; }
};

// Per-observer description of a batch (device copy in BatchCtx::obs).
struct ObsDev {
    uint32_t width, height, tiles_x, tile_base;
    uint32_t pix_base, pyr_base, has_cam64, star_tile_base;  // star_tile_base: first 16x16 star tile
    uint32_t lw[SR_BLOOM_LEVELS + 1], lh[SR_BLOOM_LEVELS + 1];
    uint32_t loff[SR_BLOOM_LEVELS + 2];  // level offsets inside this observer's pyramid
};

// A captured batch sequence, replayed while the batch's shape is unchanged.
struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

struct FastCtx {
    int num_sms = 148;
    int max_smem = 0;
    // Batch buffers, grown on demand.
    // shadow: one byte per pixel, the main light's shadow ray as traced (0 none, 1 clear, 2 occluded)
    // sched: the tile counters of the trace kernel, one per SM band then the shared pool's
    DevMem U, cam64, cam, obs, lvl_pre, hits, slots, shadow, hdr, rgb, sched;
    // Star binning: per (observer, star) cone events and tile rectangles; per 16x16 tile a count,
    // a list offset and a fill cursor; the lists; the prefix sum's scratch.
    DevMem star_cd, star_cu, star_rect, star_count, star_offset, star_fill, star_list, star_scan;
    // Gradient: the camera and the stars' cone events as duals, per-block partial sums, the result.
    DevMem adj_cam, adj_stars, adj_partials, adj_out, adj_pyr, adj_weight, adj_grid, adj_pass, adj_hdr;
    // The outcomes of the last gradient call (hits, shadows, star lists, grid lines, cut passes)
    // stay valid for frozen evaluations while no other frame is rendered.
    bool adj_valid = false;
    uint32_t adj_w = 0, adj_h = 0, adj_level = 0, adj_r0 = 0, adj_r1 = 0;  // the last gradient call's frame and band
    const float4* adj_geoms = nullptr;
    HostMem hU, hcam64, hobs, hlvl;
    uint32_t cap_obs = 0;
    std::map<uint64_t, GraphEntry> graphs;
};

cudaError_t fast_init(FastCtx& c, const cudaDeviceProp& prop);
void fast_release(FastCtx& c);
// Builds the layout from the device copy of the reference nodes. The scene is usable on the fast
// path when its depth is <= 60 (the reference's stack never overflows), it has fewer than 2^25
// primitives and every leaf holds at most 63 (the packed references); otherwise `usable` is false.
cudaError_t fast_build(FastCtx& c, FastScene& s, const SrGpuNode* nodes, uint32_t num_nodes, uint32_t depth,
                       uint32_t num_prims, uint32_t max_leaf, cudaStream_t st);
SrTuning fast_default_tuning(const FastCtx& c);
bool fast_tuning_valid(const FastCtx& c, const SrTuning& t);

// One batch of observers through the fast path.
struct BatchRequest {
    uint32_t n;
    const SrGpuUniforms* u;       // host, n entries
    const SrCameraF64* cam64;     // host, n entries or null
    uint32_t* rgb;                // device, sum of the observers' pixels (concatenated), or null (internal)
    uint32_t* hit_id;             // device, optional (same indexing as rgb)
    float* lambda;                // device, optional
    float* tau;                   // device, optional
    bool count_work;
    bool use_graph;
    bool star_brute;              // sum every star per pixel (no binning), as the reference
    cudaEvent_t* ev;              // optional: 5 events, after camera, trace, shading, stars, bloom
};
cudaError_t fast_render_batch(FastCtx& c, const FastScene& s, const SrTuning& t, const SceneDev& sd,
                              const double anchor[4], const BBConst& bb, uint32_t* counters, const BatchRequest& r,
                              cudaStream_t st);
// The gradient of sum((P_level(HDR) - P_level(target))^2) with respect to (rapidity, event) of one
// observer (see sr_adjoint.cuh). `target`: device, W*H*4 floats. out: loss, grad[7], primal
// mismatches (pixels whose dual value differs from the forward frame, or whose star list was not
// sortable), star terms. `frozen`: only the loss at `cam` under the last gradient call's discrete
// outcomes (no forward frame; the finite-difference check of the gradient). Only rows
// [row0, row1) of the loss level count (and the frame's pixel rows under them): the results of a
// partition of the rows sum to the whole frame's.
cudaError_t fast_adjoint(FastCtx& c, const FastScene& s, const SrTuning& t, const SceneDev& sd, const double anchor[4],
                         const BBConst& bb, uint32_t* counters, const SrGpuUniforms& u, const SrCameraF64& cam,
                         const float* target, uint32_t level, bool frozen, uint32_t row0, uint32_t row1,
                         double out[10], cudaStream_t st);
// The device HDR image (level 0) of observer `i` of the last batch, for side outputs.
float4* fast_batch_hdr(FastCtx& c, uint32_t pix_base_of_obs);

}  // namespace srk
