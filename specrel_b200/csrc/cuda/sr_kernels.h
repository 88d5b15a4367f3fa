// Device data of a scene and a frame, and the host-side launchers of every kernel.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/specrel.h"

namespace srk {

// Blackbody constants of star.rs:171-180 (powi(5) of the primaries and the white-point Planck
// values), computed once on the host.
struct BBConst {
    float r5, g5, b5, wr, wg, wb;
};

// A scene on the device: the reference's packed arrays plus the B200 node layout.
struct SceneDev {
    const SrGpuNode* nodes;
    const float4* geoms;          // 5 float4 per primitive, leaf order
    const float4* attrs;          // 12 float4 per primitive, leaf order
    const float4* mats;           // 3 float4 per material
    const float4* stars;          // headers then segments (gpu.rs:106-119)
    const uint32_t* leaf_to_orig; // may be null
    const uint32_t* tables;       // gamma LUT then glyph rows
    const uint4* wide;            // B200 node layout (see sr_fast.cu), may be null
    uint32_t num_nodes, num_prims, num_mats, num_stars;
    uint32_t root_is_leaf;        // the whole scene is one leaf
    uint32_t pad[3];
};

// Per-frame outputs and scratch on the device.
struct FrameDev {
    float4* hdr;         // the HDR image and its bloom pyramid (bloom.rs's layout)
    uint32_t* rgb;       // packed 0x00RRGGBB
    uint32_t* hit_id;    // optional
    float* lambda;       // optional
    float* tau;          // optional
    uint32_t* counters;  // [0] shadow rays, [1] error flags, [2] work counter, [3] spare
    uint32_t width, height;
};

// Error flag bits in counters[1].
constexpr uint32_t ERR_TRAVERSAL_LIMIT = 1u;
constexpr uint32_t ERR_BAD_MATERIAL = 2u;
constexpr uint32_t ERR_BAD_INDEX = 4u;
// The fast path's shading asked for a main-light shadow result the trace kernel did not produce
// (the two evaluate the same condition; a mismatch is an internal error).
constexpr uint32_t ERR_SHADOW_MISMATCH = 8u;

// Star binning of the fast path (sr_stars.cuh): tile side in pixels, and whether an observer's
// stars are binned. The binning assumes a field of view within a 76-degree
// half diagonal and pixels finer than 0.042 radians; other observers sum every star per pixel.
constexpr uint32_t STAR_TILE = 16;
__host__ __device__ inline bool stars_binned_for(const SrGpuUniforms& U, uint32_t num_stars) {
    if (U.mode != 0u || num_stars == 0u || U.size[1] == 0u) return false;
    const float hw = U.half_wh[0], hh = U.half_wh[1];
    const float pitch = 2.0f * hh / (float)U.size[1];
    return hw * hw + hh * hh <= 16.0f && 2.4f * pitch <= 0.1f;
}

// Pyramid geometry of bloom.rs:28-49 for one frame.
struct Pyramid {
    uint32_t w[SR_BLOOM_LEVELS + 1], h[SR_BLOOM_LEVELS + 1], off[SR_BLOOM_LEVELS + 2];
};
Pyramid make_pyramid(uint32_t width, uint32_t height);

// The plain path: one thread per pixel, the reference's traversal, shading, shadows and stars.
cudaError_t launch_render_plain(const SceneDev& s, const SrGpuUniforms& u, const float4* cam_dev, const FrameDev& f,
                                const BBConst& bb, cudaStream_t st);
// FP64 observer: builds the tetrad from a rapidity in double precision, rebases the event to the
// scene anchor, rounds to f32 and writes 6 float4 (event, e0..e3, frontier origin) to `cam_dev`.
cudaError_t launch_camera_f64(const SrCameraF64& c, const double anchor[4], const SrGpuUniforms& u, float4* cam_dev,
                              cudaStream_t st);
// Bvh4D::trace and interpolate_hit of caller rays (sr_trace_rays), the reference's traversal;
// error flags into counters[1].
cudaError_t launch_trace_rays(const SceneDev& s, const double anchor[4], const SrRay* rays, uint32_t n, SrRayHit* hits,
                              uint32_t* counters, cudaStream_t st);
// Bloom pyramid, composite, tone map and pack into f.rgb.
cudaError_t launch_bloom(const FrameDev& f, const Pyramid& p, const uint32_t* tables, cudaStream_t st);

}  // namespace srk
