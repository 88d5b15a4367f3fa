// BVH build on the GPU (sr_build.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/specrel.h"

namespace srk {

struct GpuBuildInfo {
    uint32_t num_nodes, depth, max_leaf;
    uint32_t unsupported;  // a split left one side empty (the reference selects by median there)
};

// Builds the reference's tree over n simplex boxes (device, build order; box i is box[2i] = min,
// box[2i + 1] = max, (t, x, y, z)): nodes (device, room for 2n) in depth-first order, order[i] =
// the build index of leaf slot i.
cudaError_t gpu_bvh_build(const float4* box, uint32_t n, SrGpuNode* nodes, uint32_t* order, GpuBuildInfo* info,
                          cudaStream_t st);

// Many independent trees in one build: segment s is the simplices [seg[s].start, + seg[s].count)
// of the build-order arrays, and its tree is the reference's tree over them alone. Its nodes go to
// nodes[tree[s].node_base, + tree[s].num_nodes) with links absolute in that array and leaves
// pointing at absolute leaf slots (its leaf slots are its own range [start, + count)), order as
// above. An empty segment has no nodes. `info` gets the totals (num_nodes: of all trees).
struct GpuSegment {
    uint32_t start, count;
};
struct GpuTreeInfo {
    uint32_t node_base, num_nodes, depth, max_leaf;
};
cudaError_t gpu_bvh_build_forest(const float4* box, uint32_t n, const GpuSegment* seg, uint32_t num_seg,
                                 SrGpuNode* nodes, uint32_t* order, GpuTreeInfo* tree, GpuBuildInfo* info,
                                 cudaStream_t st);

// Keeps the current device's stream-ordered pool from returning memory at synchronisation (once).
cudaError_t keep_build_pool();

// The simplices of worldtubes (build order) extruded on the device: records and boxes in device
// buffers from the stream-ordered pool that the caller frees (cudaFreeAsync on the same stream),
// num_prims of them. With `tube_first` (host, num_tubes + 1 entries), tube b's simplices are
// [tube_first[b], tube_first[b + 1]). rindler_bad: some tube of two samples or more has a vertex
// with 1 + a_local . p <= 0 at some sample (the reference asserts against it).
struct ExtrudeOut {
    SrGpuGeom* geoms;
    SrGpuAttr* attrs;
    float4* boxes;
    uint32_t num_prims;
    uint32_t rindler_bad;
};
cudaError_t gpu_extrude(const SrTube* tubes, uint32_t num_tubes, ExtrudeOut* out, cudaStream_t st,
                        uint32_t* tube_first = nullptr);

// Hot and cold records from build order into leaf order (out[i] = in[order[i]]).
cudaError_t gpu_gather_records(const uint32_t* order, uint32_t n, const SrGpuGeom* gin, const SrGpuAttr* ain,
                               SrGpuGeom* gout, SrGpuAttr* aout, cudaStream_t st);

}  // namespace srk
