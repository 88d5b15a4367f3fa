"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liboracle_specrel.so).

The oracle is a C++ restatement of the reference's CPU renderer (src/renderer.rs, bvh4d.rs,
mesh4d.rs, star.rs, bloom.rs, minkowski.rs), templated on float (the reference's f32 path)
and double (the FP64 oracle). Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, always as the checker or the timed CPU baseline, never as a product
code path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_specrel.so")


def build(force: bool = False) -> None:
    """Compile the oracle library and its known-answer test program (make, g++)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)


class SynthParams(C.Structure):
    _fields_ = [("config", C.c_uint32), ("n_bodies", C.c_uint32), ("steps", C.c_uint32),
                ("subdiv", C.c_uint32), ("n_stars", C.c_uint32), ("pad", C.c_uint32),
                ("seed", C.c_uint64), ("translate", C.c_double * 4)]


class SceneInfo(C.Structure):
    _fields_ = [("n_prims", C.c_uint64), ("n_nodes", C.c_uint64), ("n_stars", C.c_uint64),
                ("n_star_vec4", C.c_uint64), ("n_materials", C.c_uint64), ("depth", C.c_uint32),
                ("rindler_ok", C.c_int32), ("superluminal", C.c_int32), ("clamped_accel", C.c_uint32),
                ("cam_pos", C.c_double * 4), ("cam_rapidity", C.c_double * 3),
                ("bounds_min", C.c_double * 4), ("bounds_max", C.c_double * 4), ("median_splits", C.c_uint32),
                ("pad", C.c_uint32)]


class Camera(C.Structure):
    _fields_ = [("pos", C.c_double * 4), ("rapidity", C.c_double * 3), ("yaw", C.c_double),
                ("pitch", C.c_double), ("roll", C.c_double), ("fov_deg", C.c_double),
                ("proper_time", C.c_double), ("use_tetrad", C.c_int32), ("pad", C.c_int32),
                ("tetrad", C.c_double * 16)]


class Config(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("mode", C.c_uint32),
                ("shadow_mode", C.c_uint32), ("slice_mode", C.c_uint32), ("prophecy_delta", C.c_float),
                ("full_height", C.c_uint32), ("row_stride", C.c_uint32), ("row_offset", C.c_uint32)]


class Flash(C.Structure):
    _fields_ = [("at", C.c_double * 4), ("width", C.c_double), ("intensity", C.c_double),
                ("color", C.c_double * 3)]


class Dynamics(C.Structure):
    _fields_ = [("has_frontier", C.c_int32), ("n_flashes", C.c_uint32), ("frontier_origin", C.c_double * 4),
                ("frontier_tau", C.c_double), ("frontier_lag", C.c_double), ("flashes", C.POINTER(Flash)),
                ("n_remote", C.c_uint32), ("pad", C.c_uint32), ("remote_origins", C.POINTER(C.c_double))]


class Observer(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("slice_mode", C.c_uint32), ("pad", C.c_uint32),
                ("pos", C.c_double * 4), ("rapidity", C.c_double * 3)]


class PixelOut(C.Structure):
    _fields_ = [("rgb", C.c_void_p), ("slot", C.c_void_p), ("orig", C.c_void_p), ("lambda_", C.c_void_p),
                ("tau", C.c_void_p), ("min_bary", C.c_void_p), ("denom_rel", C.c_void_p), ("hdr", C.c_void_p),
                ("stats", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.orc_scene_new.restype = C.c_void_p
        L.orc_scene_new.argtypes = [C.POINTER(SynthParams), C.c_int]
        L.orc_scene_free.argtypes = [C.c_void_p]
        L.orc_scene_from_packed.restype = C.c_void_p
        L.orc_scene_from_packed.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                            C.c_uint32, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
        L.orc_scene_info.argtypes = [C.c_void_p, C.POINTER(SceneInfo)]
        L.orc_scene_demo.restype = C.c_void_p
        L.orc_scene_demo.argtypes = [C.c_uint32, C.c_int]
        L.orc_scene_demo_info.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_light_clock_bounce_fraction.restype = C.c_float
        L.orc_light_clock_bounce_fraction.argtypes = [C.c_float, C.c_float]
        L.orc_material.argtypes = [C.c_uint32, C.c_void_p]
        L.orc_tetrad_from_beta.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_bvh_from_boxes.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint32)]
        L.orc_select_nth.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]
        L.orc_scene_pack.argtypes = [C.c_void_p] + [C.c_void_p] * 6
        L.orc_render.argtypes = [C.c_void_p, C.POINTER(Camera), C.POINTER(Config), C.POINTER(Dynamics),
                                 C.c_int, C.c_int, C.POINTER(PixelOut)]
        L.orc_observers.argtypes = [C.c_uint64, C.c_uint32, C.POINTER(Observer)]
        L.orc_tetrad.argtypes = [C.POINTER(Camera), C.c_int, C.POINTER(C.c_double)]
        L.orc_gamma_lut.argtypes = [C.c_void_p]
        L.orc_bloom_pack.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        L.orc_frozen_new.restype = C.c_void_p
        L.orc_frozen_new.argtypes = [C.c_void_p, C.POINTER(Camera), C.POINTER(Config), C.c_int, C.c_int]
        L.orc_frozen_free.argtypes = [C.c_void_p]
        L.orc_frozen_loss.restype = C.c_double
        L.orc_frozen_loss.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Camera), C.POINTER(Config), C.c_void_p,
                                      C.c_uint32, C.c_int, C.c_void_p]
        L.orc_arena_new.restype = C.c_void_p
        L.orc_arena_new.argtypes = []
        L.orc_arena_free.argtypes = [C.c_void_p]
        L.orc_arena_begin.argtypes = [C.c_void_p]
        L.orc_arena_tube.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32,
                                     C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
        L.orc_arena_piece.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int64, C.c_void_p,
                                      C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        L.orc_arena_finish.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_arena_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_arena_dirty.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_void_p,
                                      C.POINTER(C.c_uint32), C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32]
        L.orc_arena_pack.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_top_tree.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.orc_tube_simplices.restype = C.c_int64
        L.orc_tube_simplices.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                         C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


# Layouts of the reference's packed GPU arrays (gpu.rs:44-100).
NODE_DTYPE = np.dtype([("min", "<f4", 4), ("max", "<f4", 4), ("right_or_first", "<u4"), ("count", "<u4"),
                       ("left", "<u4"), ("pad", "<u4")])
GEOM_DTYPE = np.dtype([("v0", "<f4", 4), ("n", "<f4", 4), ("b1", "<f4", 4), ("b2", "<f4", 4), ("b3", "<f4", 4)])
ATTR_DTYPE = np.dtype([(k, "<f4", 4) for k in ("uv_u", "uv_v", "tb_x", "tb_y", "tb_z", "tau", "grad_u", "grad_v",
                                              "normal", "four_vel", "misc", "decided_at")])
MAT_DTYPE = np.dtype([("base", "<f4", 4), ("checker", "<f4", 4), ("params", "<f4", 4)])
assert NODE_DTYPE.itemsize == 48 and GEOM_DTYPE.itemsize == 80 and ATTR_DTYPE.itemsize == 192
assert MAT_DTYPE.itemsize == 48


def synth_params(config: int, seed: int, n_bodies: int | None = None, steps: int | None = None,
                 subdiv: int = 2, n_stars: int | None = None, translate=(0.0, 0.0, 0.0, 0.0)) -> SynthParams:
    """Default parameters of the five synthetic workloads."""
    p = SynthParams()
    p.config = config
    p.seed = seed
    p.n_bodies = 64 if n_bodies is None else n_bodies
    p.steps = (128 if config == 2 else 64) if steps is None else steps
    p.subdiv = subdiv
    p.n_stars = (100000 if config == 5 else 0) if n_stars is None else n_stars
    tr = (1e6, 6e4, 0.0, 8e4) if (config == 3 and tuple(translate) == (0.0, 0.0, 0.0, 0.0)) else translate
    for k in range(4):
        p.translate[k] = tr[k]
    return p


class Scene:
    """An oracle-built scene (float or double)."""

    def __init__(self, params: SynthParams | None, fp64: bool = False, _handle=None):
        self.params = params
        self.fp64 = fp64
        self.h = _handle if _handle is not None else lib().orc_scene_new(C.byref(params), 1 if fp64 else 0)
        self._free = lib().orc_scene_free  # held so that freeing works during interpreter exit
        self.info = SceneInfo()
        lib().orc_scene_info(self.h, C.byref(self.info))

    @classmethod
    def from_packed(cls, nodes, geoms, attrs, mats, stars, num_stars, light_pos=(0.0, 0.0, 50.0, 0.0)):
        """An oracle scene holding exactly the given packed arrays (gpu.rs layouts)."""
        keep = [np.ascontiguousarray(a) for a in (nodes, geoms, attrs, mats, stars)]
        lp = np.asarray(light_pos, np.float32)
        nstar_vec4 = len(keep[4]) // 4 if num_stars else 0
        h = lib().orc_scene_from_packed(keep[0].ctypes.data, len(nodes), keep[1].ctypes.data, keep[2].ctypes.data,
                                        len(geoms), keep[3].ctypes.data, len(mats), keep[4].ctypes.data, nstar_vec4,
                                        num_stars, lp.ctypes.data)
        return cls(None, False, _handle=h)

    @classmethod
    def demo(cls, which: int, fp64: bool = False):
        """One of the reference's demo scenes (scene.rs:283-720): DEMO_* below. Sets `window`
        (t_min, t_max), `light` (x, y, z) and `initial_camera` (the scene's camera event)."""
        h = lib().orc_scene_demo(which, 1 if fp64 else 0)
        if not h:
            raise ValueError(f"no demo scene {which}")
        sc = cls(None, fp64, _handle=h)
        d = np.zeros(5)
        lib().orc_scene_demo_info(h, d.ctypes.data)
        sc.window = (float(d[0]), float(d[1]))
        sc.light = (float(d[2]), float(d[3]), float(d[4]))
        sc.initial_camera = tuple(float(x) for x in sc.info.cam_pos)
        return sc

    def trace(self, rays) -> np.ndarray:
        """Bvh4D::trace (bvh4d.rs:445-520) of rays (n x 10: origin t,x,y,z, direction, t_min, t_max)
        and the interpolated hit: n x 18 (found, slot, original index, lambda, proper time,
        event t,x,y,z, tet barycentrics (4), uv (2), material)."""
        r = np.ascontiguousarray(np.atleast_2d(rays), np.float64)
        out = np.zeros((len(r), 18))
        lib().orc_trace(self.h, r.ctypes.data, len(r), out.ctypes.data)
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self._free(self.h)
            self.h = None

    def pack(self):
        """The reference's packed GPU arrays (nodes, geoms, attrs, materials, stars, order)."""
        i = self.info
        nodes = np.zeros(i.n_nodes, NODE_DTYPE)
        geoms = np.zeros(i.n_prims, GEOM_DTYPE)
        attrs = np.zeros(i.n_prims, ATTR_DTYPE)
        mats = np.zeros(i.n_materials, MAT_DTYPE)
        stars = np.zeros(max(1, i.n_star_vec4) * 4, np.float32)
        order = np.zeros(i.n_prims, np.uint32)
        rc = lib().orc_scene_pack(self.h, nodes.ctypes.data, geoms.ctypes.data, attrs.ctypes.data,
                                  mats.ctypes.data, stars.ctypes.data, order.ctypes.data)
        if rc != 0:
            raise RuntimeError("only float scenes pack")
        return nodes, geoms, attrs, mats, stars, order


DEMO_TWIN_PARADOX, DEMO_BARN_AND_POLE, DEMO_TERRELL_PENROSE_STREET, DEMO_EINSTEIN_TRAIN, DEMO_CAROUSEL = range(5)
PENROSE_SPHERE = 5  # the scene of scene.rs's Penrose silhouette test (not a demo scene)


def tetrad_from_beta(beta) -> np.ndarray:
    """Tetrad::from_beta in f32 (minkowski.rs:437-441): rows e0..e3, columns (t, x, y, z)."""
    b = np.asarray(beta, np.float64)
    out = np.zeros(16)
    lib().orc_tetrad_from_beta(b.ctypes.data, out.ctypes.data)
    return out.reshape(4, 4).astype(np.float32)


def bvh_from_boxes(boxes):
    """Bvh4D::build over boxes (n x 8: min then max, (t, x, y, z)): (nodes, order, median splits)."""
    b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 8)
    n = len(b)
    nodes = np.zeros(max(1, 2 * n - 1), NODE_DTYPE)
    order = np.zeros(max(1, n), np.uint32)
    nn, med = C.c_uint32(), C.c_uint32()
    lib().orc_bvh_from_boxes(b.ctypes.data, n, nodes.ctypes.data, order.ctypes.data, C.byref(nn), C.byref(med))
    return nodes[:nn.value], order[:n], med.value


def select_nth(keys, k):
    """The oracle's slice::select_nth_unstable_by on float keys: (keys, original positions) after."""
    v = np.ascontiguousarray(keys, np.float32).copy()
    idx = np.arange(len(v), dtype=np.uint32)
    lib().orc_select_nth(v.ctypes.data, idx.ctypes.data, len(v), k)
    return v, idx


def light_clock_bounce_fraction(proper_time: float, cavity_length: float) -> float:
    """renderer.rs:988-996 in f32."""
    return float(lib().orc_light_clock_bounce_fraction(proper_time, cavity_length))


def material(i: int) -> dict:
    """Material i of the scenes' table (scene.rs:181-275), as f32 values."""
    v = np.zeros(9)
    pattern = lib().orc_material(i, v.ctypes.data)
    return dict(base=tuple(v[0:3]), emission=v[3], checker=tuple(v[4:7]), grid_scale=v[7], cavity_length=v[8],
                pattern=pattern)


@dataclass
class RenderResult:
    rgb: np.ndarray
    slot: np.ndarray | None = None
    orig: np.ndarray | None = None
    lam: np.ndarray | None = None
    tau: np.ndarray | None = None
    min_bary: np.ndarray | None = None
    denom_rel: np.ndarray | None = None
    hdr: np.ndarray | None = None
    stats: np.ndarray | None = None


def make_camera(pos=(0, 0, 0, 0), rapidity=(0, 0, 0), fov_deg=90.0, yaw=0.0, pitch=0.0, roll=0.0,
                proper_time=0.0, tetrad=None) -> Camera:
    c = Camera()
    for k in range(4):
        c.pos[k] = pos[k]
    for k in range(3):
        c.rapidity[k] = rapidity[k]
    c.yaw, c.pitch, c.roll = yaw, pitch, roll
    c.fov_deg = fov_deg
    c.proper_time = proper_time
    if tetrad is not None:
        c.use_tetrad = 1
        flat = np.asarray(tetrad, np.float64).reshape(16)
        for k in range(16):
            c.tetrad[k] = flat[k]
    return c


def make_config(width, height, mode=0, shadow_mode=0, slice_mode=0, prophecy_delta=3.5, full_height=0,
                row_stride=1, row_offset=0) -> Config:
    """RenderConfig; with full_height > 0 only rows row_offset + k * row_stride of a full_height-row
    frame are rendered (height of them), the CPU baseline's bounded sample."""
    cf = Config()
    cf.width, cf.height, cf.mode, cf.shadow_mode, cf.slice_mode = width, height, mode, shadow_mode, slice_mode
    cf.prophecy_delta = prophecy_delta
    cf.full_height, cf.row_stride, cf.row_offset = full_height, row_stride, row_offset
    return cf


@dataclass
class DynamicsSpec:
    frontier: tuple | None = None          # (origin(4), proper_time)
    flashes: list = field(default_factory=list)  # (at(4), width, intensity, color(3))
    frontier_lag: float = 0.0
    remote_origins: list = field(default_factory=list)


def _dynamics(spec: DynamicsSpec | None):
    if spec is None:
        return None, []
    d = Dynamics()
    keep = []
    if spec.frontier is not None:
        d.has_frontier = 1
        for k in range(4):
            d.frontier_origin[k] = spec.frontier[0][k]
        d.frontier_tau = spec.frontier[1]
    d.frontier_lag = spec.frontier_lag
    if spec.flashes:
        arr = (Flash * len(spec.flashes))()
        for i, (at, w, inten, col) in enumerate(spec.flashes):
            for k in range(4):
                arr[i].at[k] = at[k]
            arr[i].width, arr[i].intensity = w, inten
            for k in range(3):
                arr[i].color[k] = col[k]
        d.flashes = arr
        d.n_flashes = len(spec.flashes)
        keep.append(arr)
    if spec.remote_origins:
        ro = np.ascontiguousarray(np.asarray(spec.remote_origins, np.float64).reshape(-1, 4))
        d.remote_origins = ro.ctypes.data_as(C.POINTER(C.c_double))
        d.n_remote = ro.shape[0]
        keep.append(ro)
    return d, keep


def render(scene: Scene, camera: Camera, cfg: Config, dynamics: DynamicsSpec | None = None, threads: int = 0,
           perturb: int = 0, aux: bool = True, hdr: bool = False, stats: bool = False) -> RenderResult:
    n = cfg.width * cfg.height
    res = RenderResult(rgb=np.zeros(n, np.uint32))
    out = PixelOut()
    out.rgb = res.rgb.ctypes.data
    if aux:
        res.slot = np.zeros(n, np.int64)
        res.orig = np.zeros(n, np.uint32)
        res.lam = np.zeros(n, np.float64)
        res.tau = np.zeros(n, np.float64)
        res.min_bary = np.zeros(n, np.float64)
        res.denom_rel = np.zeros(n, np.float64)
        out.slot, out.orig, out.lambda_ = res.slot.ctypes.data, res.orig.ctypes.data, res.lam.ctypes.data
        out.tau, out.min_bary, out.denom_rel = res.tau.ctypes.data, res.min_bary.ctypes.data, res.denom_rel.ctypes.data
    if hdr:
        res.hdr = np.zeros(n * 3, np.float64)
        out.hdr = res.hdr.ctypes.data
    if stats:
        res.stats = np.zeros(n * 4, np.uint64)
        out.stats = res.stats.ctypes.data
    d, keep = _dynamics(dynamics)
    if threads <= 0:
        threads = os.cpu_count() or 1
    rc = lib().orc_render(scene.h, C.byref(camera), C.byref(cfg), C.byref(d) if d is not None else None,
                          threads, perturb, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"orc_render failed ({rc})")
    if res.hdr is not None:
        res.hdr = res.hdr.reshape(n, 3)
    if res.stats is not None:
        res.stats = res.stats.reshape(n, 4)
    return res


def tetrad(camera: Camera, fp64: bool = False) -> np.ndarray:
    out = (C.c_double * 16)()
    lib().orc_tetrad(C.byref(camera), 1 if fp64 else 0, out)
    return np.array(out[:], np.float64).reshape(4, 4)


def observers(seed: int, n: int):
    arr = (Observer * n)()
    lib().orc_observers(seed, n, arr)
    return [dict(width=o.width, height=o.height, slice_mode=o.slice_mode, pos=tuple(o.pos[:4]),
                 rapidity=tuple(o.rapidity[:3])) for o in arr]


def gamma_lut() -> np.ndarray:
    out = np.zeros(4096, np.uint8)
    lib().orc_gamma_lut(out.ctypes.data)
    return out


def bloom_pack(hdr3: np.ndarray, w: int, h: int):
    src = np.ascontiguousarray(hdr3, np.float32).reshape(-1)
    rgb = np.zeros(w * h, np.uint32)
    bloomed = np.zeros(w * h * 3, np.float32)
    lib().orc_bloom_pack(src.ctypes.data, w, h, rgb.ctypes.data, bloomed.ctypes.data)
    return rgb, bloomed.reshape(-1, 3)


class Frozen:
    """The frame's discrete outcomes at one observer (hits, shadows, textures, sky grid lines, the
    stars passing the footprint cut), for evaluating the image loss at nearby observers with them
    held fixed: the FP64 reference for the engine's gradient (shaded, past light cone)."""

    def __init__(self, scene: Scene, camera: Camera, cfg: Config, threads: int = 0, binning: int = -1):
        """`binning`: find each pixel's candidate stars by projecting the stars (-1: on star sets
        above 4096, 0: never, 1: always); the recorded outcomes are the same either way."""
        self.scene, self.cfg = scene, cfg
        self.h = lib().orc_frozen_new(scene.h, C.byref(camera), C.byref(cfg), threads or (os.cpu_count() or 1),
                                      binning)
        self._free = lib().orc_frozen_free
        if not self.h:
            raise RuntimeError("orc_frozen_new: only shaded past-light-cone frames")

    def __del__(self):
        if getattr(self, "h", None):
            self._free(self.h)
            self.h = None

    def loss(self, camera: Camera, target: np.ndarray, level: int = 0, threads: int = 0, hdr: bool = False):
        """sum((P(HDR) - P(target))^2), P = `level` 2x2-box halvings; target: (w*h, 3) float64."""
        t = np.ascontiguousarray(target, np.float64).reshape(-1)
        out = np.zeros(t.size, np.float64) if hdr else None
        L = lib().orc_frozen_loss(self.scene.h, self.h, C.byref(camera), C.byref(self.cfg), t.ctypes.data, level,
                                  threads or (os.cpu_count() or 1), out.ctypes.data if hdr else None)
        return (L, out.reshape(-1, 3)) if hdr else L


TRI_DTYPE = np.dtype([("idx", "<u4", 3), ("uv", "<f4", (3, 2)), ("normal", "<f4", 3)])
SAMPLE_DTYPE = np.dtype([("center", "<f4", 4), ("tetrad", "<f4", (4, 4)), ("proper_time", "<f4"), ("phi", "<f4", 3),
                         ("accel", "<f4", 3), ("pad", "<f4")])


class Arena:
    """The reference's scene cache over an arena (oracle_arena.hpp): the same calls as the engine's
    sr_arena_* entry points; arrays() gives the arena's packed arrays, free room included."""

    STAT_KEYS = ("chunks_built", "chunks_reused", "simplices_built", "simplices_reused", "arena_simplices", "compacted")

    def __init__(self):
        self.h = lib().orc_arena_new()
        self._free = lib().orc_arena_free

    def __del__(self):
        if getattr(self, "h", None):
            self._free(self.h)
            self.h = None

    def begin(self):
        lib().orc_arena_begin(self.h)

    def tube(self, part, vertices, triangles, samples, material, decided=None):
        v = np.ascontiguousarray(vertices, np.float32)
        t = np.ascontiguousarray(triangles, TRI_DTYPE)
        s = np.ascontiguousarray(samples, SAMPLE_DTYPE)
        d = None if decided is None else np.ascontiguousarray(decided, np.float32)
        r = lib().orc_arena_tube(self.h, part[0], part[1], part[2], v.ctypes.data, len(v), t.ctypes.data, len(t),
                                 s.ctypes.data, len(s), None if d is None else d.ctypes.data, material)
        if r != 0:
            raise ValueError("bad tube")

    def piece(self, part, index, key, boxes, geoms, attrs):
        k = np.ascontiguousarray(key, np.uint32)
        b = np.ascontiguousarray(boxes, np.float32)
        g = np.ascontiguousarray(geoms, GEOM_DTYPE)
        a = np.ascontiguousarray(attrs, ATTR_DTYPE)
        lib().orc_arena_piece(self.h, part[0], part[1], part[2], index, k.ctypes.data, len(k), b.ctypes.data,
                              g.ctypes.data, a.ctypes.data, len(g))

    def finish(self, boxes=None, geoms=None, attrs=None) -> dict:
        st = np.zeros(6, np.uint64)
        if geoms is None or not len(geoms):
            lib().orc_arena_finish(self.h, None, None, None, 0, st.ctypes.data)
        else:
            b = np.ascontiguousarray(boxes, np.float32)
            g = np.ascontiguousarray(geoms, GEOM_DTYPE)
            a = np.ascontiguousarray(attrs, ATTR_DTYPE)
            lib().orc_arena_finish(self.h, b.ctypes.data, g.ctypes.data, a.ctypes.data, len(g), st.ctypes.data)
        return dict(zip(self.STAT_KEYS, (int(x) for x in st)))

    def dirty(self):
        """(layout, edit, node ranges, prim ranges): the arena's version and what its latest edit
        wrote (Bvh4D::version / dirty)."""
        lay, ed = C.c_uint64(), C.c_uint64()
        nn, npr = C.c_uint32(), C.c_uint32()
        lib().orc_arena_dirty(self.h, C.byref(lay), C.byref(ed), None, C.byref(nn), None, C.byref(npr), 0)
        cap = max(nn.value, npr.value, 1)
        nr = np.zeros(2 * cap, np.uint64)
        pr = np.zeros(2 * cap, np.uint64)
        lib().orc_arena_dirty(self.h, C.byref(lay), C.byref(ed), nr.ctypes.data, C.byref(nn), pr.ctypes.data,
                              C.byref(npr), cap)
        pairs = lambda a, n: [(int(a[2 * i]), int(a[2 * i + 1])) for i in range(n)]
        return lay.value, ed.value, pairs(nr, nn.value), pairs(pr, npr.value)

    def arrays(self):
        nn, npr = C.c_uint32(), C.c_uint32()
        lib().orc_arena_sizes(self.h, C.byref(nn), C.byref(npr))
        nodes = np.zeros(nn.value, NODE_DTYPE)
        geoms = np.zeros(npr.value, GEOM_DTYPE)
        attrs = np.zeros(npr.value, ATTR_DTYPE)
        lib().orc_arena_pack(self.h, nodes.ctypes.data, geoms.ctypes.data, attrs.ctypes.data)
        return nodes, geoms, attrs


def tube_simplices(vertices, triangles, samples, material, decided=None):
    """A whole tube extruded at once: boxes (n x 8), hot and cold records, in build order."""
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, TRI_DTYPE)
    s = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    d = None if decided is None else np.ascontiguousarray(decided, np.float32)
    cap = 3 * len(t) * max(len(s) - 1, 0)
    boxes = np.zeros((max(cap, 1), 8), np.float32)
    geoms = np.zeros(max(cap, 1), GEOM_DTYPE)
    attrs = np.zeros(max(cap, 1), ATTR_DTYPE)
    n = lib().orc_tube_simplices(v.ctypes.data, len(v), t.ctypes.data, len(t), s.ctypes.data, len(s),
                                 None if d is None else d.ctypes.data, material, boxes.ctypes.data, geoms.ctypes.data,
                                 attrs.ctypes.data)
    if n < 0:
        raise ValueError("bad tube")
    return boxes[:n], geoms[:n], attrs[:n]


def top_tree(boxes, roots, weights, base):
    """top_tree (bvh4d.rs:593-644): the n - 1 nodes over n subtrees, in the reference's order."""
    b = np.ascontiguousarray(boxes, np.float32)
    r = np.ascontiguousarray(roots, np.uint32)
    w = np.ascontiguousarray(weights, np.float32)
    out = np.zeros(len(r) - 1, NODE_DTYPE)
    lib().orc_top_tree(b.ctypes.data, r.ctypes.data, w.ctypes.data, len(r), base, out.ctypes.data)
    return out
