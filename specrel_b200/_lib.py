"""ctypes binding of libspecrel_cuda.so (include/specrel.h and include/specrel_scene.h).

The library is the product: the sm_100a render engine behind the C ABI plus the caller-side
host helpers. This module only loads it and declares the signatures. There is no fallback:
if the library is missing, importing the package raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspecrel_cuda.so")

# ---- status codes (specrel.h) -----------------------------------------------------------------
SR_OK = 0
SR_ERR_INVALID_ARGUMENT = 1
SR_ERR_CUDA = 2
SR_ERR_OUT_OF_MEMORY = 3
SR_ERR_NO_DEVICE = 4
SR_ERR_NO_SCENE = 5
SR_ERR_BAD_SCENE = 6
SR_ERR_TRAVERSAL_LIMIT = 7
SR_ERR_UNSUPPORTED = 8

SR_PATH_PLAIN = 0
SR_PATH_FAST = 1
SR_FLAG_TIMING = 1
SR_FLAG_DEVICE_OUTPUT = 2
SR_FLAG_STAR_BRUTE = 4
SR_FLAG_COUNT_WORK = 8
SR_FLAG_ASYNC_OUTPUT = 16
SR_NOALLOC_SCRATCH_BYTES = 8 << 20
SR_ADJ_FROZEN = 1
SR_NOALLOC_MAX_PIXELS = 1 << 18
SR_MAX_FLASHES = 16
SR_LAYOUT_AUTO, SR_LAYOUT_OCTANT, SR_LAYOUT_COMPACT = 0, 1, 2

# ---- packed layouts (gpu.rs:44-144) ------------------------------------------------------------
NODE_DTYPE = np.dtype([("min", "<f4", 4), ("max", "<f4", 4), ("right_or_first", "<u4"), ("count", "<u4"),
                       ("left", "<u4"), ("pad", "<u4")])
GEOM_DTYPE = np.dtype([("v0", "<f4", 4), ("n", "<f4", 4), ("b1", "<f4", 4), ("b2", "<f4", 4), ("b3", "<f4", 4)])
ATTR_DTYPE = np.dtype([(k, "<f4", 4) for k in ("uv_u", "uv_v", "tb_x", "tb_y", "tb_z", "tau", "grad_u", "grad_v",
                                              "normal", "four_vel", "misc", "decided_at")])
MAT_DTYPE = np.dtype([("base", "<f4", 4), ("checker", "<f4", 4), ("params", "<f4", 4)])
TRI_DTYPE = np.dtype([("idx", "<u4", 3), ("uv", "<f4", (3, 2)), ("normal", "<f4", 3)])  # SrTubeTriangle
SAMPLE_DTYPE = np.dtype([("center", "<f4", 4), ("tetrad", "<f4", (4, 4)), ("proper_time", "<f4"), ("phi", "<f4", 3),
                         ("accel", "<f4", 3), ("pad", "<f4")])  # SrTubeSample


class Ray(C.Structure):  # SrRay
    _fields_ = [("origin", C.c_double * 4), ("dir", C.c_float * 4), ("t_min", C.c_float), ("t_max", C.c_float)]


class RayHit(C.Structure):  # SrRayHit
    _fields_ = [("id", C.c_uint32), ("slot", C.c_uint32), ("lambda_", C.c_float), ("proper_time", C.c_float),
                ("event", C.c_double * 4), ("tet_bary", C.c_float * 4), ("uv", C.c_float * 2), ("material", C.c_uint32),
                ("pad", C.c_uint32)]


class GpuUniforms(C.Structure):
    _fields_ = [("cam_pos", C.c_float * 4), ("e", (C.c_float * 4) * 4), ("light_pos", C.c_float * 4),
                ("half_wh", C.c_float * 2), ("size", C.c_uint32 * 2), ("mode", C.c_uint32),
                ("shadow_mode", C.c_uint32), ("slice_mode", C.c_uint32), ("num_nodes", C.c_uint32),
                ("frontier_origin", C.c_float * 4), ("frontier_view_offset", C.c_float), ("num_flashes", C.c_uint32),
                ("frontier_tau", C.c_float), ("prophecy_delta", C.c_float), ("num_haze", C.c_uint32),
                ("num_stars", C.c_uint32), ("pad", C.c_uint32 * 2), ("haze_origin", (C.c_float * 4) * 5),
                ("flash_at", (C.c_float * 4) * 16), ("flash_col_width", (C.c_float * 4) * 16)]


class SceneDesc(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("num_nodes", C.c_uint32), ("num_prims", C.c_uint32),
                ("geoms", C.c_void_p), ("attrs", C.c_void_p), ("materials", C.c_void_p),
                ("num_materials", C.c_uint32), ("num_stars", C.c_uint32), ("stars", C.c_void_p),
                ("num_star_vec4", C.c_uint64), ("light_pos", C.c_float * 4), ("leaf_to_orig", C.c_void_p),
                ("anchor", C.c_void_p)]


class BuildDesc(C.Structure):
    _fields_ = [("boxes", C.c_void_p), ("geoms", C.c_void_p), ("attrs", C.c_void_p), ("num_prims", C.c_uint32),
                ("materials", C.c_void_p), ("num_materials", C.c_uint32), ("num_stars", C.c_uint32),
                ("stars", C.c_void_p), ("num_star_vec4", C.c_uint64), ("light_pos", C.c_float * 4),
                ("anchor", C.c_void_p)]


class Tube(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("num_vertices", C.c_uint32), ("num_triangles", C.c_uint32),
                ("triangles", C.c_void_p), ("samples", C.c_void_p), ("num_samples", C.c_uint32),
                ("material", C.c_uint32), ("decided_at", C.c_void_p)]


class ArenaPart(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("player", C.c_uint32), ("id", C.c_uint64)]


class ArenaStats(C.Structure):
    _fields_ = [("chunks_built", C.c_uint32), ("chunks_reused", C.c_uint32), ("simplices_built", C.c_uint64),
                ("simplices_reused", C.c_uint64), ("arena_simplices", C.c_uint64), ("compacted", C.c_uint32),
                ("num_nodes", C.c_uint32), ("bvh_depth", C.c_uint32), ("rindler_crossed", C.c_uint32)]


class Range(C.Structure):
    _fields_ = [("start", C.c_uint64), ("end", C.c_uint64)]


class Timings(C.Structure):
    _fields_ = [("submit_ms", C.c_float), ("wait_ms", C.c_float), ("kernel_ms", C.c_float),
                ("readback_ms", C.c_float), ("camera_ms", C.c_float), ("trace_ms", C.c_float),
                ("shade_ms", C.c_float), ("stars_ms", C.c_float), ("bloom_ms", C.c_float),
                ("shadow_rays", C.c_uint32), ("pad", C.c_uint32),
                ("nodes_visited", C.c_uint64), ("leaves_visited", C.c_uint64), ("tets_tested", C.c_uint64),
                ("shadow_nodes_visited", C.c_uint64), ("shadow_leaves_visited", C.c_uint64),
                ("shadow_tets_tested", C.c_uint64)]


class Outputs(C.Structure):
    _fields_ = [("rgb", C.c_void_p), ("hit_id", C.c_void_p), ("lambda_", C.c_void_p), ("tau", C.c_void_p),
                ("hdr", C.c_void_p)]


class CameraF64(C.Structure):
    _fields_ = [("event", C.c_double * 4), ("rapidity", C.c_double * 3), ("yaw", C.c_double),
                ("pitch", C.c_double), ("roll", C.c_double)]


class RenderOpts(C.Structure):
    _fields_ = [("path", C.c_uint32), ("flags", C.c_uint32), ("cam64", C.POINTER(CameraF64))]


class SceneStats(C.Structure):
    _fields_ = [("num_nodes", C.c_uint32), ("num_prims", C.c_uint32), ("num_stars", C.c_uint32),
                ("bvh_depth", C.c_uint32), ("device_bytes", C.c_uint64), ("fast_nodes", C.c_uint32),
                ("rindler_crossed", C.c_uint32), ("box_copies", C.c_uint32), ("pad", C.c_uint32)]


class AdjointResult(C.Structure):
    _fields_ = [("loss", C.c_double), ("grad", C.c_double * 7), ("primal_mismatch", C.c_double),
                ("star_terms", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("tile_w", C.c_uint32),
                ("tile_h", C.c_uint32), ("chunk_tiles", C.c_uint32), ("refill_lanes", C.c_uint32),
                ("leaf_coop", C.c_uint32), ("leaf_batch", C.c_uint32),
                ("home_pct", C.c_uint32), ("stack_smem", C.c_uint32), ("top_levels", C.c_uint32),
                ("packet", C.c_uint32)]


class SynthParams(C.Structure):
    _fields_ = [("config", C.c_uint32), ("n_bodies", C.c_uint32), ("steps", C.c_uint32), ("subdiv", C.c_uint32),
                ("n_stars", C.c_uint32), ("threads", C.c_uint32), ("seed", C.c_uint64),
                ("translate", C.c_double * 4)]


class SynthInfo(C.Structure):
    _fields_ = [("bvh_depth", C.c_uint32), ("rindler_ok", C.c_int32), ("clamped_accel", C.c_uint32),
                ("max_leaf", C.c_uint32), ("cam_pos", C.c_double * 4), ("cam_rapidity", C.c_double * 3),
                ("anchor", C.c_double * 4), ("build_seconds", C.c_double), ("median_splits", C.c_uint32),
                ("pad", C.c_uint32)]


class ObserverDraw(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("slice_mode", C.c_uint32), ("pad", C.c_uint32),
                ("pos", C.c_double * 4), ("rapidity", C.c_double * 3)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 4), ("e", (C.c_float * 4) * 4), ("proper_time", C.c_float),
                ("fov_y_rad", C.c_float)]


class RenderConfig(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("mode", C.c_uint32), ("shadow_mode", C.c_uint32),
                ("slice_mode", C.c_uint32), ("prophecy_delta", C.c_float)]


class Flash(C.Structure):
    _fields_ = [("at", C.c_float * 4), ("width", C.c_float), ("intensity", C.c_float), ("color", C.c_float * 3)]


class FrameDynamics(C.Structure):
    _fields_ = [("has_frontier", C.c_int32), ("n_flashes", C.c_uint32), ("frontier_origin", C.c_float * 4),
                ("frontier_tau", C.c_float), ("frontier_lag", C.c_float), ("flashes", C.POINTER(Flash)),
                ("remote_origins", C.POINTER(C.c_float)), ("n_remote", C.c_uint32), ("pad", C.c_uint32)]


assert C.sizeof(GpuUniforms) == 768 and C.sizeof(Timings) == 96

_lib = None

# Every function either header declares, with its ctypes signature.
# sr_sum_f64_fn: the caller's sum over a group (0 on success).
SUM_F64_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_size_t, C.c_void_p)


class NcclSum(C.Structure):  # SrNcclSum
    _fields_ = [("comm", C.c_void_p), ("stream", C.c_void_p), ("device_buf", C.c_void_p)]


SIGNATURES = {
    "sr_create": (C.c_int32, [C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "sr_destroy": (None, [C.c_void_p]),
    "sr_last_error": (C.c_char_p, [C.c_void_p]),
    "sr_adapter_name": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sr_set_stream": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "sr_synchronize": (C.c_int32, [C.c_void_p]),
    "sr_scene_validate": (C.c_int32, [C.POINTER(SceneDesc), C.POINTER(C.c_uint32), C.c_char_p, C.c_size_t]),
    "sr_upload_scene": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(SceneDesc)]),
    "sr_build_scene": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(BuildDesc)]),
    "sr_scene_tree": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                  C.POINTER(C.c_uint32)]),
    "sr_scene_boxes": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "sr_scene_tubes": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint32)]),
    "sr_top_tree": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                C.POINTER(C.c_uint32)]),
    "sr_build_scene_tubes": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(BuildDesc)]),
    "sr_arena_begin": (C.c_int32, [C.c_void_p, C.c_uint32]),
    "sr_arena_tube": (C.c_int32, [C.c_void_p, C.c_uint32, ArenaPart, C.POINTER(Tube)]),
    "sr_arena_reuse": (C.c_int32, [C.c_void_p, C.c_uint32, ArenaPart, C.c_int64, C.c_void_p, C.c_uint32,
                                   C.POINTER(C.c_int32)]),
    "sr_arena_install": (C.c_int32, [C.c_void_p, C.c_uint32, ArenaPart, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_uint32]),
    "sr_arena_finish": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(BuildDesc), C.POINTER(ArenaStats)]),
    "sr_scene_records": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32]),
    "sr_update_scene": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(SceneDesc), C.POINTER(Range), C.c_uint32,
                                    C.POINTER(Range), C.c_uint32]),
    "sr_scene_stats": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(SceneStats)]),
    "sr_set_layout": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "sr_render": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.c_void_p, C.c_uint64,
                              C.POINTER(Timings)]),
    "sr_render_ex": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.POINTER(RenderOpts),
                                 C.POINTER(Outputs), C.POINTER(Timings)]),
    "sr_render_batch": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.POINTER(CameraF64),
                                    C.c_uint32, C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(Timings)]),
    "sr_adjoint": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.POINTER(CameraF64), C.c_void_p,
                               C.c_uint32, C.c_uint32, C.POINTER(AdjointResult)]),
    "sr_adjoint_rows": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.POINTER(CameraF64), C.c_void_p,
                                    C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(AdjointResult)]),
    "sr_trace_rays": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]),
    "sr_adjoint_band": (C.c_int32, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]),
    "sr_adjoint_reduce": (C.c_int32, [C.POINTER(AdjointResult), SUM_F64_FN, C.c_void_p]),
    "sr_adjoint_group": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.POINTER(CameraF64), C.c_void_p,
                                     C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, SUM_F64_FN, C.c_void_p,
                                     C.POINTER(AdjointResult)]),
    "sr_nccl_sum_f64": (C.c_int, [C.POINTER(C.c_double), C.c_size_t, C.c_void_p]),
    "sr_render_noalloc": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.POINTER(CameraF64), C.c_void_p]),
    "sr_get_tuning": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(Tuning)]),
    "sr_set_tuning": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(Tuning)]),
    "sr_autotune": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(GpuUniforms), C.c_uint32, C.POINTER(Tuning),
                                C.POINTER(C.c_float)]),
    "sr_scene_synth": (C.c_int32, [C.POINTER(SynthParams), C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "sr_scene_free": (None, [C.c_void_p]),
    "sr_bvh_build_host": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "sr_scene_desc": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc)]),
    "sr_scene_info": (C.c_int32, [C.c_void_p, C.POINTER(SynthInfo)]),
    "sr_observers_synth": (C.c_int32, [C.c_uint64, C.c_uint32, C.POINTER(ObserverDraw)]),
    "sr_camera_new": (C.c_int32, [C.POINTER(C.c_float), C.c_float, C.POINTER(Camera)]),
    "sr_camera_boost_local": (C.c_int32, [C.POINTER(Camera), C.POINTER(C.c_float)]),
    "sr_camera_rotate_local": (C.c_int32, [C.POINTER(Camera), C.c_float, C.c_float, C.c_float]),
    "sr_uniforms_build": (C.c_int32, [C.POINTER(Camera), C.POINTER(RenderConfig), C.POINTER(FrameDynamics),
                                      C.c_uint32, C.POINTER(C.c_float), C.c_uint32, C.POINTER(GpuUniforms)]),
    "sr_tables_build": (C.c_int32, [C.POINTER(C.c_uint32)]),
    "sr_flash_emit": (C.c_int32, [C.POINTER(Flash), C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.c_int]),
    "sr_flashes_retire": (C.c_int32, [C.POINTER(Flash), C.POINTER(C.c_uint32), C.c_float]),
    "sr_flashes_shift_time": (C.c_int32, [C.POINTER(Flash), C.c_uint32, C.c_float]),
    "sr_config_step_prophecy_delta": (C.c_int32, [C.POINTER(RenderConfig), C.c_float]),
}


def lib():
    """Load the library (raises if it has not been built: there is no other implementation)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
                              "(or __graft_entry__.build()); the engine has no fallback path")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class SrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"status {status}: {msg}")
        self.status = status
