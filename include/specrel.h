/*
 * specrel.h — C ABI of the B200 render engine for SpecRel's per-pixel render path.
 *
 * It replaces the wgpu backend `GpuRenderer` (src/gpu.rs:432-901) behind the same data split the
 * reference already uses: static scene arrays uploaded once (`PackedSceneGpuData`,
 * src/gpu.rs:232-315) and a 768-byte per-frame uniform block (`GpuUniforms`,
 * src/gpu.rs:122-212). A Rust caller binds these functions with `extern "C"` and `#[repr(C)]`
 * mirrors of the structs below (their sizes and offsets are fixed by the static_asserts at the
 * end of this header) and keeps `Scene4D::build`, `PackedSceneGpuData::from_scene` and
 * `GpuUniforms::build` as they are.
 *
 * Conventions: every function returns an `sr_status` (no aborts); host buffers belong to the
 * caller, device buffers to the context; one CUDA stream per context; a context is not
 * thread-safe (the reference's `&mut self`).
 */
#ifndef SPECREL_H
#define SPECREL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SR_MAX_FLASHES 16        /* renderer.rs:179 */
#define SR_MAX_HAZE_ORIGINS 5    /* renderer.rs:224 */
#define SR_GAMMA_LUT_SIZE 4096   /* renderer.rs:1102 */
#define SR_BLOOM_LEVELS 6        /* bloom.rs:23 */
#define SR_STACK_SIZE 64         /* bvh4d.rs:454, :537 */

/* ---- Packed scene arrays, byte for byte the reference's layouts ---------------------------- */

/* GpuNode (gpu.rs:44-51). Leaf when count > 0 (right_or_first = first hot record); else an
 * internal node with children `left` and `right_or_first`. 4-vectors are (t, x, y, z). */
typedef struct SrGpuNode {
    float min[4];
    float max[4];
    uint32_t right_or_first;
    uint32_t count;
    uint32_t left;
    uint32_t pad;
} SrGpuNode;

/* GpuGeom (gpu.rs:68-74): the 80-byte hot record of SimplexGeom4D (mesh4d.rs:153-159). */
typedef struct SrGpuGeom {
    float v0[4];
    float n[4];
    float b1[4];
    float b2[4];
    float b3[4];
} SrGpuGeom;

/* GpuAttr (gpu.rs:79-92): cold attributes, transposed (one row = one component, 4 vertices).
 * misc = (uv_world_scale.u, uv_world_scale.v, bitcast<f32>(material_id), 0). */
typedef struct SrGpuAttr {
    float uv_u[4], uv_v[4];
    float tb_x[4], tb_y[4], tb_z[4];
    float tau[4];
    float grad_u[4], grad_v[4];
    float normal[4];
    float four_vel[4];
    float misc[4];
    float decided_at[4];
} SrGpuAttr;

/* GpuMaterial (gpu.rs:96-100): base = (rgb, emission), checker = (rgb, grid_scale),
 * params = (wireframe_width, bitcast<f32>(pattern), cavity_length, 0). */
typedef struct SrGpuMaterial {
    float base[4];
    float checker[4];
    float params[4];
} SrGpuMaterial;

/* GpuUniforms (gpu.rs:122-144), 768 bytes. */
typedef struct SrGpuUniforms {
    float cam_pos[4];
    float e[4][4];
    float light_pos[4];
    float half_wh[2];
    uint32_t size[2];
    uint32_t mode;         /* 0 shaded, 1 isochrones, 2 tetrahedron inspector, 3 decision age */
    uint32_t shadow_mode;  /* 0 off, 1 Lorentz-invariant (null), 2 camera slice */
    uint32_t slice_mode;   /* 0 past light cone, 1 God's-eye slice, 2 frontier, 3 prophecy */
    uint32_t num_nodes;
    float frontier_origin[4];
    float frontier_view_offset;
    uint32_t num_flashes;
    float frontier_tau;
    float prophecy_delta;
    uint32_t num_haze;
    uint32_t num_stars;
    uint32_t pad[2];
    float haze_origin[SR_MAX_HAZE_ORIGINS][4];
    float flash_at[SR_MAX_FLASHES][4];
    float flash_col_width[SR_MAX_FLASHES][4];
} SrGpuUniforms;

/* PackedSceneGpuData (gpu.rs:232-244) plus two optional sidecars. */
typedef struct SrSceneDesc {
    const SrGpuNode* nodes;
    uint32_t num_nodes;
    uint32_t num_prims;
    const SrGpuGeom* geoms;           /* num_prims, leaf order */
    const SrGpuAttr* attrs;           /* num_prims, leaf order */
    const SrGpuMaterial* materials;
    uint32_t num_materials;
    uint32_t num_stars;               /* star headers at the front of `stars` */
    const float* stars;               /* pack_stars (gpu.rs:106-119), num_star_vec4 x vec4 */
    uint64_t num_star_vec4;
    float light_pos[4];               /* (unused, x, y, z) */
    /* Optional: leaf slot -> original simplex index (Bvh4D::order, bvh4d.rs:72-73), so hit ids
     * are reported in the caller's simplex order; NULL reports leaf slots. */
    const uint32_t* leaf_to_orig;
    /* Optional: FP64 anchor (t, x, y, z) that every f32 coordinate of the scene is relative to;
     * NULL means the origin. Used by the FP64 camera path (sr_render_ex with `cam64`). */
    const double* anchor;
} SrSceneDesc;

typedef struct SrRange { uint64_t start, end; } SrRange;

/* ---- Status ------------------------------------------------------------------------------- */
typedef int32_t sr_status;
#define SR_OK 0
#define SR_ERR_INVALID_ARGUMENT 1
#define SR_ERR_CUDA 2
#define SR_ERR_OUT_OF_MEMORY 3
#define SR_ERR_NO_DEVICE 4
#define SR_ERR_NO_SCENE 5
#define SR_ERR_BAD_SCENE 6
#define SR_ERR_TRAVERSAL_LIMIT 7
#define SR_ERR_UNSUPPORTED 8

typedef struct sr_ctx sr_ctx;

/* GpuTimings (gpu.rs:408-420), milliseconds, plus per-phase device times recorded with CUDA
 * events on the context's stream when SR_FLAG_TIMING is set. */
typedef struct SrTimings {
    float submit_ms;
    float wait_ms;
    float kernel_ms;    /* whole frame on the device */
    float readback_ms;
    float camera_ms;    /* FP64 camera / rebase kernel */
    float trace_ms;     /* primary traversal (+ shading for the plain path; + the main
                           light's shadow rays for the fast path) */
    float shade_ms;     /* shading, with the flashes' shadow rays (fast path) */
    float stars_ms;     /* star cone events, binning and gather */
    float bloom_ms;     /* bloom pyramid + tone map + pack */
    uint32_t shadow_rays;
    uint32_t pad;
    /* Traversal work, filled when SR_FLAG_COUNT_WORK is set (a slower counting variant of the
     * kernels): internal-node visits (each tests two child boxes), leaf visits and tetrahedron
     * tests, for primary rays and for shadow rays. */
    uint64_t nodes_visited, leaves_visited, tets_tested;
    uint64_t shadow_nodes_visited, shadow_leaves_visited, shadow_tets_tested;
} SrTimings;

/* Which implementation renders a frame. */
#define SR_PATH_PLAIN 0   /* one thread per pixel, the reference's BVH2 traversal order */
#define SR_PATH_FAST 1    /* persistent traversal over the B200 node layout, per-lane ray fetch */

#define SR_FLAG_TIMING 1u          /* record per-phase CUDA events into SrTimings */
#define SR_FLAG_DEVICE_OUTPUT 2u   /* output pointers are device pointers; return without syncing */
#define SR_FLAG_STAR_BRUTE 4u      /* stars: O(N_stars) per pixel as the reference, no binning */
#define SR_FLAG_COUNT_WORK 8u      /* count traversal work into SrTimings (slower; blocks) */
#define SR_FLAG_ASYNC_OUTPUT 16u   /* sr_render_batch with a host framebuffer: return once the batch
                                      and its readback are queued; the readback runs beside the next
                                      batch. The framebuffer holds the frames after sr_synchronize
                                      (or after the call two batches later returns), which also
                                      reports a device error of the batch. Not with timings. */

/* Optional per-pixel outputs (host or device pointers, as the call's flags say). */
typedef struct SrOutputs {
    uint32_t* rgb;      /* W*H packed 0x00RRGGBB (required) */
    uint32_t* hit_id;   /* W*H original simplex index of the primary hit, 0xFFFFFFFF on a miss */
    float* lambda;      /* W*H affine parameter of the primary hit */
    float* tau;         /* W*H interpolated proper time of the primary hit */
    float* hdr;         /* W*H*4 pre-bloom radiance (r, g, b, 0) */
} SrOutputs;

/* The observer in FP64: event and tetrad are built on the GPU in double precision, rebased to the
 * scene anchor, then rounded to the f32 uniforms the traversal uses. */
typedef struct SrCameraF64 {
    double event[4];      /* (t, x, y, z) in world coordinates */
    double rapidity[3];   /* Tetrad::rest().boost_local(rapidity) (minkowski.rs:467-479) */
    double yaw, pitch, roll;  /* then rotate_local (minkowski.rs:498-521) */
} SrCameraF64;

typedef struct SrRenderOpts {
    uint32_t path;               /* SR_PATH_* */
    uint32_t flags;              /* SR_FLAG_* */
    const SrCameraF64* cam64;    /* optional FP64 camera (overrides cam_pos / e of the uniforms) */
} SrRenderOpts;

/* ---- Context ----------------------------------------------------------------------------- */

/* GpuRenderer::new (gpu.rs:472-620), device half: picks CUDA device `device`, creates the stream,
 * uploads the gamma LUT and glyph tables (gpu.rs:223-229). */
sr_status sr_create(int device, sr_ctx** out, char* err, size_t errlen);
void sr_destroy(sr_ctx* ctx);
const char* sr_last_error(const sr_ctx* ctx);
/* GpuRenderer::adapter_name (gpu.rs:734). */
sr_status sr_adapter_name(const sr_ctx* ctx, char* buf, size_t len);
/* Use a caller-owned cudaStream_t (NULL: the context's own stream). */
sr_status sr_set_stream(sr_ctx* ctx, void* cuda_stream);
sr_status sr_synchronize(sr_ctx* ctx);

/* ---- Scenes ------------------------------------------------------------------------------ */

/* GpuRenderer::upload_scene (gpu.rs:622-699): copies the packed arrays to the device, validates
 * them (child links, leaf ranges, material ids) and builds the B200 node layout on the device. */
sr_status sr_upload_scene(sr_ctx* ctx, uint32_t scene_idx, const SrSceneDesc* desc);
/* Whether a node is BvhNode4D::NOTHING (bvh4d.rs:31): interior, both links to node 0, and an
 * empty box. As the root it makes the scene's tree empty (an arena before anything is written). */
#define SR_NODE_IS_NOTHING(n)                                                                   \
    ((n)->count == 0 && (n)->left == 0 && (n)->right_or_first == 0 &&                              \
     ((n)->min[0] > (n)->max[0] || (n)->min[1] > (n)->max[1] || (n)->min[2] > (n)->max[2] ||       \
      (n)->min[3] > (n)->max[3]))
/* The host-side checks sr_upload_scene runs before copying (no device needed): child links and
 * leaf ranges in bounds, every node reached once from the root, material ids, leaf_to_orig and
 * star segment ranges in bounds. `depth` (optional) receives the tree depth. The reference's
 * upload (gpu.rs:622-699) trusts its own builder and has no counterpart. */
sr_status sr_scene_validate(const SrSceneDesc* desc, uint32_t* depth, char* err, size_t errlen);
/* GpuRenderer::update_scene (gpu.rs:704-731): writes only the dirty node and primitive ranges
 * when they fit the arrays already on the device, else uploads afresh. `desc` holds the full
 * new arrays; the ranges say which items changed since the last upload or update. */
sr_status sr_update_scene(sr_ctx* ctx, uint32_t scene_idx, const SrSceneDesc* desc, const SrRange* node_ranges,
                          uint32_t n_node_ranges, const SrRange* prim_ranges, uint32_t n_prim_ranges);

/* The simplices of a scene in build order, for the build on the device. */
typedef struct SrBuildDesc {
    const float* boxes;               /* num_prims x 8: box min (t, x, y, z), then max (t, x, y, z) */
    const SrGpuGeom* geoms;           /* num_prims, build order */
    const SrGpuAttr* attrs;           /* num_prims, build order */
    uint32_t num_prims;
    const SrGpuMaterial* materials;
    uint32_t num_materials;
    uint32_t num_stars;
    const float* stars;               /* as SrSceneDesc */
    uint64_t num_star_vec4;
    float light_pos[4];
    const double* anchor;             /* optional, as SrSceneDesc */
} SrBuildDesc;
/* Bvh4D::build (bvh4d.rs:123-141, 287-427) and the leaf-order packing of
 * PackedSceneGpuData::from_scene (gpu.rs:247-289) run on the device: the tree over the simplices'
 * boxes (8-bin SAH over the four axes, the reference's partition order), the hot and cold records
 * gathered into leaf order, then the B200 node layout. The node array and leaf order are those of
 * the host build. Hit ids are reported in build order (the tree's leaf order is kept as
 * leaf_to_orig). A split that leaves one side empty, where the reference selects by median,
 * returns SR_ERR_UNSUPPORTED (build such a scene on the host and use sr_upload_scene). A scene
 * already at the index is replaced, its device buffers reused when large enough (a scene rebuilt
 * every frame allocates nothing once warm); after a failed build the index holds no scene. */
sr_status sr_build_scene(sr_ctx* ctx, uint32_t scene_idx, const SrBuildDesc* desc);
/* Worldtubes for the build on the device: a body's mesh swept along its sampled worldline
 * (extend_worldtube_simplices, mesh4d.rs:721-854), static geometry unless per-sample causal
 * decision stamps are given (build_worldtube_simplices_with_decided, mesh4d.rs:648-660). */
typedef struct SrTubeTriangle {       /* Triangle3D (mesh4d.rs:438-443) */
    uint32_t idx[3];
    float uv[3][2];
    float normal[3];                  /* (x, y, z) */
} SrTubeTriangle;
typedef struct SrTubeSample {         /* WorldlineSample (mesh4d.rs:615-630) */
    float center[4];                  /* (t, x, y, z) */
    float tetrad[4][4];               /* e0..e3, each (t, x, y, z) */
    float proper_time;
    float phi[3];                     /* proper-time gradient in the body frame */
    float accel[3];                   /* proper acceleration in the body frame */
    float pad;
} SrTubeSample;
typedef struct SrTube {
    const float* vertices;            /* num_vertices x (x, y, z), body frame */
    uint32_t num_vertices;
    uint32_t num_triangles;
    const SrTubeTriangle* triangles;
    const SrTubeSample* samples;
    uint32_t num_samples;
    uint32_t material;
    const float* decided_at;          /* num_samples stamps (tetrahedron corners on sample k get
                                         decided_at[k]), or NULL: static geometry (-1e9) */
} SrTube;
/* The whole scene build on the device: the worldtubes' simplices (Simplex4D::new, mesh4d.rs:312-371,
 * the Dompierre split of each triangle between consecutive samples, degenerate tetrahedra skipped)
 * in tube order, then the tree and packing of sr_build_scene. `rest` supplies materials, stars,
 * light_pos and anchor (its boxes, geoms and attrs are not used). The records equal the host
 * builder's bit for bit. A tube that crosses its Rindler horizon (1 + a_local . p <= 0 for a
 * vertex at a sample, where the reference asserts, mesh4d.rs:738-751) is extruded all the same,
 * as the host builder does, and flagged in SrSceneStats.rindler_crossed. */
sr_status sr_build_scene_tubes(sr_ctx* ctx, uint32_t scene_idx, const SrTube* tubes, uint32_t num_tubes,
                               const SrBuildDesc* rest);
/* The device scene's node array and leaf order (leaf slot -> build index) read back. Either buffer
 * may be NULL; `num_nodes` receives the node count. No counterpart in the reference (its tree
 * lives on the host). */
sr_status sr_scene_tree(sr_ctx* ctx, uint32_t scene_idx, SrGpuNode* nodes, uint32_t nodes_cap, uint32_t* order,
                        uint32_t order_cap, uint32_t* num_nodes);
/* The device scene's hot and cold records (leaf order) read back; either buffer may be NULL. */
sr_status sr_scene_records(sr_ctx* ctx, uint32_t scene_idx, SrGpuGeom* geoms, SrGpuAttr* attrs, uint32_t cap);

/* ---- Incremental scenes: the scene cache over a device arena -------------------------------
 * SceneCache (dynamic/scene_cache.rs:120-356) with the arena edits of Bvh4D (bvh4d.rs:168-215,
 * 583-644), the arena living in the scene's device arrays. A snapshot is cut into chunks, each a
 * BVH of its own; a chunk whose inputs equal the previous snapshot's keeps its nodes and records
 * where they are, the others are extruded (tubes) and built (all of a snapshot's new chunks in one
 * device build) into free room of the arrays, and a tree over the chunks' roots (top_tree) goes to
 * node 0 and free room. Once the free room exceeds half the live slots plus 16384, the chunks are
 * moved together first (compaction, no BVH build). The node array, hot and cold records equal the
 * reference's arena byte for byte. Hit ids are arena slots (the arena's leaf order is the
 * identity). The scene at `scene_idx` renders as it was until sr_arena_finish, which makes the
 * new snapshot live. A slot that does not hold this cache's arena starts afresh. */
typedef struct SrArenaPart {          /* Part (scene_cache.rs:39-44) */
    uint32_t kind;                    /* 0 body, 1 hull, 2 pulse */
    uint32_t player;
    uint64_t id;                      /* body uid, or pulse sequence number */
} SrArenaPart;
typedef struct SrArenaStats {         /* CacheStats (scene_cache.rs:59-70) */
    uint32_t chunks_built, chunks_reused;
    uint64_t simplices_built, simplices_reused;
    uint64_t arena_simplices;         /* simplex slots in use or free */
    uint32_t compacted;
    uint32_t num_nodes;               /* node slots in use or free */
    uint32_t bvh_depth;
    uint32_t rindler_crossed;         /* a new chunk's tube crosses its Rindler horizon (see below) */
} SrArenaStats;
/* SceneCache::begin: start a snapshot into the arena at `scene_idx`. */
sr_status sr_arena_begin(sr_ctx* ctx, uint32_t scene_idx);
/* SceneCache::tube: `tube` in chunks of 1.0 lab time (by each segment's first sample, the sample at
 * a boundary shared by both chunks); a chunk made from the same bits as last snapshot's is reused,
 * the others are made in sr_arena_finish. The mesh's full contents stand for the reference's hash
 * of it in the chunk's key. */
sr_status sr_arena_tube(sr_ctx* ctx, uint32_t scene_idx, SrArenaPart part, const SrTube* tube);
/* SceneCache::piece in two steps: `reused` is 1 when chunk (part, index) was last made from the
 * same `key`; when 0, give its simplices (build order, as SrBuildDesc) with sr_arena_install
 * before sr_arena_finish (a chunk never installed is empty). A chunk used twice in one snapshot is
 * an error. */
sr_status sr_arena_reuse(sr_ctx* ctx, uint32_t scene_idx, SrArenaPart part, int64_t index, const uint32_t* key,
                         uint32_t key_len, int32_t* reused);
sr_status sr_arena_install(sr_ctx* ctx, uint32_t scene_idx, SrArenaPart part, int64_t index, const float* boxes,
                           const SrGpuGeom* geoms, const SrGpuAttr* attrs, uint32_t num_prims);
/* SceneCache::finish: chunks unused this snapshot are dropped, new chunks built on the device and
 * written, `desc`'s simplices (the volatile part, may be empty) built afresh as one more chunk,
 * the tree over all chunks written, and the B200 node layout rebuilt; materials, stars, light
 * and anchor come from `desc`. `stats` (optional) receives the snapshot's CacheStats. A failure
 * before the arena is written (invalid input) undoes the snapshot: the scene and the cache are as
 * they were, and so they are after a snapshot begun and never finished; a later failure (device
 * memory) leaves no scene at the index, and the next snapshot starts afresh. A tube crossing its
 * Rindler horizon (1 + a_local . p <= 0 for a vertex at a sample, mesh4d.rs:738-751, where the
 * reference asserts) is extruded all the same, as the host builders do, and flagged in
 * `rindler_crossed`. */
sr_status sr_arena_finish(sr_ctx* ctx, uint32_t scene_idx, const SrBuildDesc* desc, SrArenaStats* stats);

typedef struct SrSceneStats {
    uint32_t num_nodes, num_prims, num_stars, bvh_depth;
    uint64_t device_bytes;
    uint32_t fast_nodes;   /* nodes of the B200 layout */
    uint32_t rindler_crossed; /* built from tubes, some vertex at some sample has 1 + a_local . p <= 0 */
    uint32_t box_copies;   /* copies of the B200 layout's child boxes: 16 (octant) or 1 (compact) */
    uint32_t pad;
} SrSceneStats;
sr_status sr_scene_stats(const sr_ctx* ctx, uint32_t scene_idx, SrSceneStats* out);

/* The fast path's node layout. SR_LAYOUT_OCTANT keeps 16 copies of every wide node's child boxes,
 * one per sign octant of a ray's inverse direction with each box's near corner first, so the slab
 * test needs no per-axis min / max (1,024 bytes of boxes per internal node of the reference tree).
 * SR_LAYOUT_COMPACT keeps one copy (64 bytes per internal node) and orders the corners per axis
 * while traversing. SR_LAYOUT_AUTO, the default, takes the octant copies when the 15 extra copies
 * need at most an eighth of the device's memory and all 16 fit in its free memory, else the
 * compact layout. Hits, lambda, tau and the nodes visited are the same in every layout. The choice
 * applies to the scene at `scene_idx` now (its layout is rebuilt) and to every later upload or
 * build at that index. */
#define SR_LAYOUT_AUTO 0u
#define SR_LAYOUT_OCTANT 1u
#define SR_LAYOUT_COMPACT 2u
sr_status sr_set_layout(sr_ctx* ctx, uint32_t scene_idx, uint32_t layout);

/* ---- Frames ------------------------------------------------------------------------------- */

/* GpuRenderer::render (gpu.rs:798-900): renders scene `scene_idx` with uniforms `u` into the
 * caller's host framebuffer (`fb_len` = width * height packed 0x00RRGGBB) and blocks until it
 * is there. Uses the fast path. */
sr_status sr_render(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, uint32_t* framebuffer,
                    uint64_t fb_len, SrTimings* timings);

/* The general form: explicit path, optional side outputs, optional FP64 camera, and (with
 * SR_FLAG_DEVICE_OUTPUT) device-resident outputs with no synchronisation. */
sr_status sr_render_ex(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, const SrRenderOpts* opts,
                       const SrOutputs* out, SrTimings* timings);

/* Many observers of one scene in one persistent launch (recorded once into a CUDA graph and
 * replayed). Observer i renders with uniforms `u[i]` (and `cam64[i]` when cam64 is not NULL)
 * into `rgb_out + offset_i`, offset_i = sum of width*height of observers before it.
 * With `timings`, the batch's device time is returned (kernel_ms); SR_FLAG_TIMING adds the
 * per-phase times and SR_FLAG_COUNT_WORK the traversal work; both run the launch sequence
 * outside its graph. */
sr_status sr_render_batch(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, const SrCameraF64* cam64,
                          uint32_t n_observers, uint32_t* rgb_out, uint64_t rgb_len, uint32_t flags,
                          SrTimings* timings);

/* ---- Ray queries ---------------------------------------------------------------------------
 * Bvh4D::trace (bvh4d.rs:445-520) followed by Simplex4D::interpolate_hit (mesh4d.rs:382-425) for
 * caller rays: the query the reference's scene probes (scene.rs:785-1053), picking and aiming make
 * on the host, here on the device with the reference's traversal order. Ray i starts at event
 * `origin` (double; rebased to the scene's FP64 anchor in double, then rounded to f32, so with no
 * anchor it is the f32 origin) and runs along `dir` over (t_min, t_max). `hits` receives, per ray,
 * the hit simplex (the caller's index through leaf_to_orig, else the leaf slot; 0xFFFFFFFF on a
 * miss), its parameter lambda, the interpolated proper time, the event (the anchor added back in
 * double), the tetrahedron barycentrics, the uv and the material. Host buffers; blocking. */
typedef struct SrRay {
    double origin[4];  /* (t, x, y, z) */
    float dir[4];
    float t_min, t_max;
} SrRay;
typedef struct SrRayHit {
    uint32_t id;    /* the hit simplex in the caller's order, or 0xFFFFFFFF */
    uint32_t slot;  /* its leaf slot, or 0xFFFFFFFF */
    float lambda, proper_time;
    double event[4];
    float tet_bary[4];
    float uv[2];
    uint32_t material, pad;
} SrRayHit;
sr_status sr_trace_rays(sr_ctx* ctx, uint32_t scene_idx, const SrRay* rays, uint32_t n, SrRayHit* hits);

/* ---- Gradient with respect to the observer ------------------------------------------------
 * New (the reference renders forward only). For one observer on the past light cone (mode 0,
 * slice mode 0, no flashes, no haze) on the fast path:
 *   loss = sum over pixels and r, g, b of (P(HDR) - P(target))^2 on the linear pre-bloom HDR
 *          image, P = `level` (0..6) halvings by 2x2 box averages (0: the image itself; the
 *          coarser levels widen the basin for a coarse-to-fine descent)
 *   grad = d loss / d (rapidity x, y, z, event t, x, y, z) of the FP64 observer `cam`
 * The forward frame's discrete outcomes (hit tetrahedra, shadow tests, textures, sky grid lines,
 * star segments and footprint cuts) are held fixed; everything smooth is differentiated in
 * forward mode in f32 with f64 accumulation. `target_hdr` is a device buffer of width*height*4
 * floats (r, g, b, unused), the layout of SrOutputs.hdr. */
typedef struct SrAdjointResult {
    double loss;
    double grad[7];
    double primal_mismatch;  /* pixels whose recomputed value differs from the forward frame (0 expected) */
    double star_terms;       /* (pixel, star) footprint terms differentiated */
} SrAdjointResult;
#define SR_ADJ_FROZEN 1u  /* only the loss at `cam`, under the discrete outcomes of the previous
                             gradient call (same scene and frame size, no frame rendered in between):
                             a smooth function of theta for checking the gradient by differences */
sr_status sr_adjoint(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, const SrCameraF64* cam,
                     const float* target_hdr, uint32_t level, uint32_t flags, SrAdjointResult* out);
/* sr_adjoint over rows [row_begin, row_end) of the loss level (`level` halvings of the frame's
 * height) and the frame's pixel rows under them: the loss terms of those rows and the gradient
 * they contribute, plus their primal mismatches and star terms. The results over a partition of the
 * rows sum to sr_adjoint's (up to the order of FP64 sums): each GPU of a group takes a band and one
 * all-reduce of the ten doubles gives the whole (the forward frame is rendered whole on each). A
 * frozen evaluation takes the rows of the gradient call before it. */
sr_status sr_adjoint_rows(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, const SrCameraF64* cam,
                          const float* target_hdr, uint32_t level, uint32_t flags, uint32_t row_begin,
                          uint32_t row_end, SrAdjointResult* out);

/* ---- The gradient over a group of GPUs ------------------------------------------------------
 * No counterpart in the reference (it renders on one device). One observer's gradient shards over
 * `world` ranks, one GPU each, every rank holding the scene and the target image: each rank
 * evaluates its band of the loss level's rows (sr_adjoint_rows) and the ten doubles of
 * SrAdjointResult are summed over the group. The sum is the caller's collective, passed in as a
 * function: an ncclAllReduce of doubles on the caller's communicator, an MPI_Allreduce, or
 * sr_nccl_sum_f64 below. It returns 0 on success. */
typedef int (*sr_sum_f64_fn)(double* values, size_t count, void* user);
/* Rank `rank`'s band of the loss level's rows (`level` halvings of `height`, rounding up, as the
 * loss takes them): [*row_begin, *row_end), contiguous, sizes differing by at most one, empty when
 * the level has fewer rows than ranks. Host only. */
sr_status sr_adjoint_band(uint32_t height, uint32_t level, uint32_t rank, uint32_t world, uint32_t* row_begin,
                          uint32_t* row_end);
/* Sums `r` (loss, gradient[7], primal mismatches, star terms) over the group in place through
 * `sum`. Host only. */
sr_status sr_adjoint_reduce(SrAdjointResult* r, sr_sum_f64_fn sum, void* user);
/* sr_adjoint_rows over this rank's band, then sr_adjoint_reduce: every rank receives the whole
 * frame's loss and gradient. Every rank of the group calls it (a rank with an empty band adds
 * zeros), in the same order relative to the caller's other collectives. `flags` as sr_adjoint (a
 * frozen evaluation follows this rank's previous gradient call). */
sr_status sr_adjoint_group(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, const SrCameraF64* cam,
                           const float* target_hdr, uint32_t level, uint32_t flags, uint32_t rank, uint32_t world,
                           sr_sum_f64_fn sum, void* user, SrAdjointResult* out);
/* A sum for sr_adjoint_reduce / sr_adjoint_group over NCCL: `user` points to an SrNcclSum. The
 * library loads NCCL (libnccl.so.2) at the first call; the caller creates the communicator, one
 * rank per GPU. The values go through `device_buf` (at least `count` doubles of device memory the
 * caller owns) on `stream`, and the call waits for them. Returns the ncclResult_t, or -1 when
 * NCCL cannot be loaded, -2 on a CUDA error. */
typedef struct SrNcclSum {
    void* comm;          /* ncclComm_t */
    void* stream;        /* cudaStream_t (NULL: the legacy default stream) */
    double* device_buf;
} SrNcclSum;
int sr_nccl_sum_f64(double* values, size_t count, void* user);

/* ---- Rendering without device allocation -------------------------------------------------
 * No counterpart in the reference: an entry point for callers that cannot call cudaMalloc while
 * they render, for instance an application whose own allocator owns all device memory under a fixed
 * budget, or a real-time loop in which cudaMalloc/cudaFree (which can synchronize the whole device)
 * would stall its other streams. sr_render_noalloc renders one frame on the plain path into the
 * caller's device buffer `rgb_dev` (width*height packed 0x00RRGGBB; `cam64` optional, as in
 * sr_render_ex) and allocates nothing: its scratch (error counters, FP64 camera rows, the HDR image
 * and its bloom pyramid) is one static device array of SR_NOALLOC_SCRATCH_BYTES that every GPU
 * which loads this library holds until the process exits.
 * - Frames above SR_NOALLOC_MAX_PIXELS pixels (e.g. 512x512 or 640x400 fit) are rejected with
 *   SR_ERR_INVALID_ARGUMENT; that is the only size rule (the scratch holds the bloom pyramid of
 *   every frame within it, one-row frames included).
 * - Every call looks up the array's device address on the current device (cudaGetSymbolAddress; the
 *   first call on a device also loads the library's device code there, if that has not happened).
 * - Every call uses the same array and leaves its contents behind (the counters are cleared at the
 *   start of each call). Calls that overlap on one GPU, from other streams or contexts of the
 *   process, race on it.
 * - The call waits for its frame (it copies the error flags back to the host and synchronizes the
 *   context's stream), so it cannot be called while that stream is being captured into a graph. */
#define SR_NOALLOC_SCRATCH_BYTES (8u << 20)
#define SR_NOALLOC_MAX_PIXELS (1u << 18)
sr_status sr_render_noalloc(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, const SrCameraF64* cam64,
                            uint32_t* rgb_dev);

/* Launch parameters of the fast path; the autotuner (sr_autotune) picks them per scene. */
typedef struct SrTuning {
    uint32_t block_threads;   /* threads per block of the persistent traversal kernel: 64..512 */
    uint32_t blocks_per_sm;   /* resident blocks per SM: 1..16 */
    uint32_t tile_w, tile_h;  /* pixel tile of 32 consecutive rays (tile_w * tile_h == 32) */
    uint32_t chunk_tiles;     /* tiles a warp takes from the frame at a time: 1..64 */
    uint32_t refill_lanes;    /* idle lanes that make a warp load new rays: 1..32 (32: all idle) */
    uint32_t leaf_coop;       /* 1: a warp tests the leaves of all its lanes together */
    uint32_t leaf_batch;      /* lanes on a leaf before the warp tests leaves: 1..32 */
    uint32_t home_pct;        /* share of the tiles (0..100) split into one band per SM, which the
                                 warps on that SM take first; the rest go in frame order */
    uint32_t stack_smem;      /* traversal-stack entries per thread kept in shared memory, 0..64
                                 (0: the whole stack in local memory); deeper entries go to local
                                 memory, so the visiting order does not depend on it */
    uint32_t top_levels;      /* levels of the wide tree staged in shared memory per block, 0..8
                                 (0: none); with stack_smem 0 or 12; the compact layout
                                 (sr_set_layout) stages none */
    uint32_t packet;          /* 1 (the default): the warp walks its tile's primary rays as one
                                 packet (one node sequence for its 32 rays, each lane with its
                                 own closest hit), then its main-light shadow rays likewise; the
                                 same hits as the per-ray order, equal-lambda ties included, as
                                 long as every hit lies beyond its leaf box's computed entry
                                 parameter (the records' 1e-4 box padding keeps a margin of
                                 1e-4 / |d| in ray parameter against its rounding); with
                                 stack_smem 0, top_levels 0 and the single-tile schedule.
                                 0: each ray walks the tree in its own near-first order (work
                                 counts, SR_FLAG_COUNT_WORK, always come from this order) */
} SrTuning;
sr_status sr_get_tuning(const sr_ctx* ctx, uint32_t scene_idx, SrTuning* out);
sr_status sr_set_tuning(sr_ctx* ctx, uint32_t scene_idx, const SrTuning* t);
/* Times candidate SrTuning values on a batch of `n` copies of the observer `u` (the batched path,
 * replayed from its captured graph after a warm-up batch), in two sweeps taking each candidate's
 * better time, and keeps the fastest for this scene; the current tuning stays unless a candidate
 * is at least 1% faster. `best_ms`: the winner's time per frame. */
sr_status sr_autotune(sr_ctx* ctx, uint32_t scene_idx, const SrGpuUniforms* u, uint32_t n, SrTuning* best,
                      float* best_ms);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
static_assert(sizeof(SrGpuNode) == 48, "GpuNode is 48 bytes (gpu.rs:44-51)");
static_assert(sizeof(SrGpuGeom) == 80, "GpuGeom is 80 bytes (gpu.rs:68-74)");
static_assert(sizeof(SrGpuAttr) == 192, "GpuAttr is 192 bytes (gpu.rs:79-92)");
static_assert(sizeof(SrTubeTriangle) == 48, "SrTubeTriangle is 48 bytes");
static_assert(sizeof(SrTubeSample) == 112, "SrTubeSample is 112 bytes");
static_assert(sizeof(SrTube) == 48, "SrTube is 48 bytes");
static_assert(sizeof(SrArenaPart) == 16 && sizeof(SrArenaStats) == 48, "arena structs");
static_assert(sizeof(SrGpuMaterial) == 48, "GpuMaterial is 48 bytes (gpu.rs:96-100)");
static_assert(sizeof(SrGpuUniforms) == 768, "GpuUniforms is 768 bytes (gpu.rs:122-144)");
static_assert(sizeof(SrTuning) == 48, "SrTuning is 12 words");
static_assert(sizeof(SrRay) == 56 && sizeof(SrRayHit) == 80, "ray query records");
static_assert(sizeof(SrAdjointResult) == 80 && sizeof(SrCameraF64) == 80, "gradient records");
static_assert(offsetof(SrGpuUniforms, light_pos) == 80, "Uniforms.light_pos");
static_assert(offsetof(SrGpuUniforms, num_nodes) == 124, "Uniforms.num_nodes");
static_assert(offsetof(SrGpuUniforms, frontier_origin) == 128, "Uniforms.frontier_origin");
static_assert(offsetof(SrGpuUniforms, frontier_view_offset) == 144, "Uniforms.frontier_view_offset");
static_assert(offsetof(SrGpuUniforms, num_flashes) == 148, "Uniforms.num_flashes");
static_assert(offsetof(SrGpuUniforms, frontier_tau) == 152, "Uniforms.frontier_tau");
static_assert(offsetof(SrGpuUniforms, num_haze) == 160, "Uniforms.num_haze");
static_assert(offsetof(SrGpuUniforms, num_stars) == 164, "Uniforms.num_stars");
static_assert(offsetof(SrGpuUniforms, haze_origin) == 176, "Uniforms.haze_origin");
static_assert(offsetof(SrGpuUniforms, flash_at) == 256, "Uniforms.flash_at");
static_assert(offsetof(SrGpuUniforms, flash_col_width) == 512, "Uniforms.flash_col_width");
static_assert(offsetof(SrGpuAttr, misc) == 160, "Attr.misc");
static_assert(offsetof(SrGpuAttr, decided_at) == 176, "Attr.decided_at");
#endif

#endif /* SPECREL_H */
