/*
 * specrel_scene.h — host-side helpers on the caller's side of the boundary, in C++.
 *
 * In the reference these steps run in Rust before the GPU backend sees any data:
 *   Scene4D::build / Bvh4D::build (scene.rs:164, bvh4d.rs:123-141) and the worldtube pipeline
 *   (mesh4d.rs:312-371, :721-854, :912-1052); PackedSceneGpuData::from_scene (gpu.rs:247-289);
 *   Camera4D / Tetrad setup (renderer.rs:45-65, minkowski.rs:424-596); GpuUniforms::build
 *   (gpu.rs:147-211).
 * This library restates them so the benchmarks and tests can produce the reference's packed
 * arrays and uniform blocks for the seeded synthetic workloads without a Rust toolchain. A Rust
 * caller keeps its own code and only binds include/specrel.h.
 */
#ifndef SPECREL_SCENE_H
#define SPECREL_SCENE_H

#include "specrel.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A seeded synthetic workload. config: 1 = 64 inertial unit cubes; 2 = 64 accelerated
 * icospheres; 3 = configuration 1 translated by `translate` (FP64 anchor); 4 = configuration 1's
 * scene (the batched-observer workload); 5 = configuration 1's scene plus `n_stars` point stars. */
typedef struct SrSynthParams {
    uint32_t config;
    uint32_t n_bodies;
    uint32_t steps;
    uint32_t subdiv;
    uint32_t n_stars;
    uint32_t threads;     /* worker threads for extrusion and the BVH build (0: all cores) */
    uint64_t seed;
    double translate[4];  /* configuration 3's offset (t, x, y, z) */
} SrSynthParams;

typedef struct sr_scene sr_scene;

typedef struct SrSynthInfo {
    uint32_t bvh_depth;
    int32_t rindler_ok;      /* the reference's f32 finite-difference check (mesh4d.rs:742-749) */
    uint32_t clamped_accel;  /* bodies whose |a| was clamped to 0.8 / r */
    uint32_t max_leaf;
    double cam_pos[4];       /* the workload's observer event */
    double cam_rapidity[3];  /* the workload's observer rapidity */
    double anchor[4];        /* FP64 anchor of the f32 coordinates */
    double build_seconds;
    uint32_t median_splits;  /* nodes split at the centroid median (bvh4d.rs:418-424): the SAH split
                                left one side empty; sr_build_scene does not take such scenes */
    uint32_t pad;
} SrSynthInfo;

/* Bvh4D::build (bvh4d.rs:123-141, 287-427) on the host from the simplices' boxes in build order (8
 * floats each: min then max, (t, x, y, z)); centroids are the box centres. `nodes` (at least 2n - 1)
 * receives the node array, `order` (n) the leaf order (leaf slot -> build index), `median_splits`
 * (optional) the number of nodes split at the centroid median, which selects as Rust's
 * slice::select_nth_unstable_by does. `threads`: worker threads for large subtrees. */
sr_status sr_bvh_build_host(const float* boxes, uint32_t n, uint32_t threads, SrGpuNode* nodes, uint32_t nodes_cap,
                            uint32_t* order, uint32_t* num_nodes, uint32_t* median_splits);

/* Builds the workload (threads: params->threads). */
sr_status sr_scene_synth(const SrSynthParams* params, sr_scene** out, char* err, size_t errlen);
void sr_scene_free(sr_scene* s);
/* Pointers into the scene's packed arrays (valid until sr_scene_free). */
sr_status sr_scene_desc(const sr_scene* s, SrSceneDesc* out);
sr_status sr_scene_info(const sr_scene* s, SrSynthInfo* out);
/* The simplices' padded boxes in build order (8 floats each: min, max, (t, x, y, z)), the input of
 * sr_build_scene; the packed arrays' leaf_to_orig maps leaf slots to this order. */
sr_status sr_scene_boxes(const sr_scene* s, const float** boxes);
/* The scene's worldtubes (meshes, samples and materials of its bodies, in build order), the input
 * of sr_build_scene_tubes (valid until sr_scene_free). */
sr_status sr_scene_tubes(const sr_scene* s, const SrTube** tubes, uint32_t* num_tubes);

/* top_tree (bvh4d.rs:593-644), on the host: the tree over n >= 2 subtrees already in an arena,
 * item i with box boxes[8i .. 8i+7] (min t, x, y, z, then max), root node roots[i], weight
 * weights[i] (its simplex count) and depth depths[i] (optional). Writes the n - 1 tree nodes to
 * `nodes` in the reference's order: the first goes to node 0, the k-th to node base + k - 1, and
 * they link to each other and to the roots accordingly. `depth` (optional) receives the depth of
 * the whole tree (tree nodes above a subtree plus its own depth). The scene cache calls it for
 * every snapshot (sr_arena_finish). */
sr_status sr_top_tree(const float* boxes, const uint32_t* roots, const float* weights, const uint32_t* depths,
                      uint32_t n, uint32_t base, SrGpuNode* nodes, uint32_t* depth);

/* One observer of the batched workload (configuration 4). */
typedef struct SrObserverDraw {
    uint32_t width, height, slice_mode, pad;
    double pos[4];
    double rapidity[3];
} SrObserverDraw;
sr_status sr_observers_synth(uint64_t seed, uint32_t n, SrObserverDraw* out);

/* Camera4D (renderer.rs:45-65) with its f32 tetrad. */
typedef struct SrCamera {
    float position[4];
    float e[4][4];
    float proper_time;
    float fov_y_rad;
} SrCamera;
/* Camera4D::new(position, fov_deg): rest tetrad, fov_deg.to_radians(). */
sr_status sr_camera_new(const float position[4], float fov_deg, SrCamera* out);
/* Tetrad::boost_local (minkowski.rs:467-479) and rotate_local (minkowski.rs:498-521). */
sr_status sr_camera_boost_local(SrCamera* cam, const float d_rapidity[3]);
sr_status sr_camera_rotate_local(SrCamera* cam, float yaw, float pitch, float roll);

/* RenderConfig (renderer.rs:160-168). */
typedef struct SrRenderConfig {
    uint32_t width, height, mode, shadow_mode, slice_mode;
    float prophecy_delta;
} SrRenderConfig;

/* FlashEvent (renderer.rs:185-190) and FrameDynamics (renderer.rs:205-218). */
typedef struct SrFlash {
    float at[4];
    float width, intensity;
    float color[3];
} SrFlash;
typedef struct SrFrameDynamics {
    int32_t has_frontier;
    uint32_t n_flashes;
    float frontier_origin[4];
    float frontier_tau;
    float frontier_lag;
    const SrFlash* flashes;
    const float* remote_origins;  /* n_remote x 4 */
    uint32_t n_remote;
    uint32_t pad;
} SrFrameDynamics;

/* The flash list of FrameDynamics (renderer.rs:179, 228, 274-311), kept by the caller in an array
 * of at least SR_MAX_FLASHES entries holding *n of them, oldest first:
 * - sr_flash_emit: FrameDynamics::emit_flash (hit = 0: width 0.8, intensity 2.5, colour
 *   (1, 0.9, 0.7)) or emit_hit_flash (hit != 0: width 0.5, intensity 3, colour (1, 0.35, 0.12))
 *   at event `at`; the oldest is evicted when SR_MAX_FLASHES are held;
 * - sr_flashes_retire: retire_flashes, keeps (in order) the flashes with now_t - at.t < 200 (the
 *   shell radius beyond which they light nothing the renderers reach);
 * - sr_flashes_shift_time: shift_time, adds dt to every flash's lab time. */
sr_status sr_flash_emit(SrFlash* flashes, uint32_t* n, const float at[4], int hit);
sr_status sr_flashes_retire(SrFlash* flashes, uint32_t* n, float now_t);
sr_status sr_flashes_shift_time(SrFlash* flashes, uint32_t n, float dt);
/* RenderConfig::step_prophecy_delta (renderer.rs:121-124, 172-175): prophecy_delta + steps * 0.5,
 * clamped to [0.5, 20]. */
sr_status sr_config_step_prophecy_delta(SrRenderConfig* cfg, float steps);

/* GpuUniforms::build (gpu.rs:147-211). `dyn` may be NULL (FrameDynamics::default()). */
sr_status sr_uniforms_build(const SrCamera* cam, const SrRenderConfig* cfg, const SrFrameDynamics* dyn,
                            uint32_t num_nodes, const float light_pos[4], uint32_t num_stars, SrGpuUniforms* out);

/* build_tables_data (gpu.rs:223-229): 4096 gamma-LUT entries then 14 glyphs x 7 rows. */
sr_status sr_tables_build(uint32_t* out4194);

#ifdef __cplusplus
}
#endif

#endif /* SPECREL_SCENE_H */
