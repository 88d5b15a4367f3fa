"""specrel_b200: B200-native engine for SpecRel's per-pixel render path.

The engine is libspecrel_cuda.so (sm_100a CUDA kernels behind the C ABI of include/specrel.h);
this package is its Python binding, used by the tests and the benchmark in the role the Rust
host code (src/gpu.rs's callers) plays in the reference:

  * ``Engine``      — GpuRenderer (gpu.rs:432-901): upload scenes, render frames, batches.
  * ``synth_scene`` — the seeded synthetic workloads, built by the library's C++ scene pipeline
                      (include/specrel_scene.h), packed as PackedSceneGpuData (gpu.rs:232-315).
  * ``camera`` / ``uniforms`` — Camera4D and GpuUniforms::build (gpu.rs:147-211).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (ATTR_DTYPE, GEOM_DTYPE, MAT_DTYPE, NODE_DTYPE, SAMPLE_DTYPE, SR_FLAG_DEVICE_OUTPUT,
                   SR_FLAG_TIMING, SR_PATH_FAST, SR_PATH_PLAIN, TRI_DTYPE, CameraF64, GpuUniforms, SrError)

__all__ = ["Engine", "PackedScene", "SynthScene", "TubeData", "synth_scene", "camera", "uniforms", "observers", "tables",
           "SR_PATH_FAST", "SR_PATH_PLAIN", "SR_FLAG_TIMING", "SR_FLAG_DEVICE_OUTPUT", "SrError", "CameraF64",
           "GpuUniforms", "validate"]


def _check(status: int, ctx=None, what: str = ""):
    if status != _lib.SR_OK:
        msg = _lib.lib().sr_last_error(ctx).decode() if ctx else what
        raise SrError(status, f"{what}: {msg}" if what and ctx else msg)


@dataclass
class PackedScene:
    """PackedSceneGpuData (gpu.rs:232-244) as numpy arrays, plus the optional sidecars."""
    nodes: np.ndarray
    geoms: np.ndarray
    attrs: np.ndarray
    materials: np.ndarray
    stars: np.ndarray          # float32, vec4 entries flattened
    num_stars: int
    light_pos: tuple = (0.0, 0.0, 50.0, 0.0)
    leaf_to_orig: np.ndarray | None = None
    anchor: tuple | None = None

    def desc(self) -> tuple[_lib.SceneDesc, list]:
        d = _lib.SceneDesc()
        keep = []

        def ptr(a):
            if a is None or a.size == 0:
                return None
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data

        d.nodes = ptr(self.nodes)
        d.num_nodes = len(self.nodes)
        d.num_prims = len(self.geoms)
        d.geoms = ptr(self.geoms)
        d.attrs = ptr(self.attrs)
        d.materials = ptr(self.materials)
        d.num_materials = len(self.materials)
        d.num_stars = self.num_stars
        d.stars = ptr(self.stars) if self.num_stars else None
        d.num_star_vec4 = (len(self.stars) // 4) if self.num_stars else 0
        for k in range(4):
            d.light_pos[k] = self.light_pos[k]
        d.leaf_to_orig = ptr(self.leaf_to_orig)
        if self.anchor is not None:
            an = np.asarray(self.anchor, np.float64)
            keep.append(an)
            d.anchor = an.ctypes.data
        return d, keep


def validate(scene: PackedScene) -> tuple[int, int, str]:
    """sr_scene_validate: (status, depth, message) without a device."""
    d, keep = scene.desc()
    depth = C.c_uint32(0)
    err = C.create_string_buffer(256)
    st = _lib.lib().sr_scene_validate(C.byref(d), C.byref(depth), err, 256)
    return st, depth.value, err.value.decode()


class SynthScene:
    """A seeded synthetic workload built by the library's C++ scene pipeline (sr_scene_synth)."""

    def __init__(self, config: int, seed: int, n_bodies: int = 64, steps: int | None = None, subdiv: int = 2,
                 n_stars: int | None = None, translate=None, threads: int = 0):
        p = _lib.SynthParams()
        p.config = config
        p.seed = seed
        p.n_bodies = n_bodies
        p.steps = (128 if config == 2 else 64) if steps is None else steps
        p.subdiv = subdiv
        p.n_stars = (100000 if config == 5 else 0) if n_stars is None else n_stars
        p.threads = threads
        tr = translate if translate is not None else ((1e6, 6e4, 0.0, 8e4) if config == 3 else (0, 0, 0, 0))
        for k in range(4):
            p.translate[k] = tr[k]
        self.params = p
        h = C.c_void_p()
        err = C.create_string_buffer(256)
        st = _lib.lib().sr_scene_synth(C.byref(p), C.byref(h), err, 256)
        if st != _lib.SR_OK:
            raise SrError(st, err.value.decode())
        self.h = h
        self._free = _lib.lib().sr_scene_free  # held so that freeing works during interpreter exit
        self.info = _lib.SynthInfo()
        _lib.lib().sr_scene_info(self.h, C.byref(self.info))
        d = _lib.SceneDesc()
        _lib.lib().sr_scene_desc(self.h, C.byref(d))
        self._desc = d

    def __del__(self):
        if getattr(self, "h", None):
            self._free(self.h)
            self.h = None

    def desc(self):
        return self._desc, [self]

    @property
    def num_nodes(self) -> int:
        return self._desc.num_nodes

    @property
    def num_prims(self) -> int:
        return self._desc.num_prims

    @property
    def num_stars(self) -> int:
        return self._desc.num_stars

    @property
    def light_pos(self):
        return tuple(self._desc.light_pos[k] for k in range(4))

    def build_inputs(self):
        """The simplices in build order, the input of Engine.build: boxes (n x 8 float32), hot and cold
        records (from the packed leaf-order arrays through leaf_to_orig)."""
        p = self.packed()
        bp = C.c_void_p()
        _check(_lib.lib().sr_scene_boxes(self.h, C.byref(bp)), what="scene_boxes")
        n = len(p.geoms)
        boxes = np.frombuffer((C.c_float * (8 * n)).from_address(bp.value), np.float32).reshape(n, 8).copy()
        geoms = np.empty_like(p.geoms)
        attrs = np.empty_like(p.attrs)
        geoms[p.leaf_to_orig] = p.geoms
        attrs[p.leaf_to_orig] = p.attrs
        return boxes, geoms, attrs, p

    def tubes(self) -> list["TubeData"]:
        """Copies of the scene's worldtubes (mesh, triangles, worldline samples, material)."""
        tp = C.c_void_p()
        nt = C.c_uint32()
        _check(_lib.lib().sr_scene_tubes(self.h, C.byref(tp), C.byref(nt)), what="scene_tubes")
        out = []
        for t in (_lib.Tube * nt.value).from_address(tp.value) if nt.value else ():
            def arr(ptr, n, dtype):
                if not n:
                    return np.zeros(0, dtype)
                return np.frombuffer((C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr), dtype).copy()
            out.append(TubeData(arr(t.vertices, 3 * t.num_vertices, np.float32).reshape(-1, 3),
                                arr(t.triangles, t.num_triangles, TRI_DTYPE), arr(t.samples, t.num_samples, SAMPLE_DTYPE),
                                int(t.material)))
        return out

    def packed(self) -> PackedScene:
        """Copies of the packed arrays as numpy (for comparisons in tests)."""
        d = self._desc

        def arr(ptr, n, dtype):
            if not n:
                return np.zeros(0, dtype)
            buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dtype, count=n).copy()

        stars = arr(d.stars, d.num_star_vec4 * 4, np.float32) if d.num_stars else np.zeros(4, np.float32)
        anchor = tuple(self.info.anchor[k] for k in range(4))
        return PackedScene(arr(d.nodes, d.num_nodes, NODE_DTYPE), arr(d.geoms, d.num_prims, GEOM_DTYPE),
                           arr(d.attrs, d.num_prims, ATTR_DTYPE), arr(d.materials, d.num_materials, MAT_DTYPE),
                           stars, d.num_stars, self.light_pos, arr(d.leaf_to_orig, d.num_prims, np.uint32), anchor)


def synth_scene(config: int, seed: int, **kw) -> SynthScene:
    return SynthScene(config, seed, **kw)


def camera(position=(0.0, 0.0, 0.0, 0.0), fov_deg: float = 90.0, rapidity=None, yaw=0.0, pitch=0.0, roll=0.0,
           proper_time: float = 0.0) -> _lib.Camera:
    """Camera4D::new then Tetrad::boost_local / rotate_local, all in f32 (renderer.rs:57-64)."""
    L = _lib.lib()
    c = _lib.Camera()
    pos = (C.c_float * 4)(*position)
    _check(L.sr_camera_new(pos, fov_deg, C.byref(c)), what="camera_new")
    if rapidity is not None and any(r != 0 for r in rapidity):
        _check(L.sr_camera_boost_local(C.byref(c), (C.c_float * 3)(*rapidity)), what="boost_local")
    if yaw or pitch or roll:
        _check(L.sr_camera_rotate_local(C.byref(c), yaw, pitch, roll), what="rotate_local")
    c.proper_time = proper_time
    return c


def uniforms(cam: _lib.Camera, width: int, height: int, mode: int = 0, shadow_mode: int = 0, slice_mode: int = 0,
             prophecy_delta: float = 3.5, num_nodes: int = 0, light_pos=(0.0, 0.0, 50.0, 0.0), num_stars: int = 0,
             frontier=None, flashes=(), frontier_lag: float = 0.0, remote_origins=()) -> GpuUniforms:
    """GpuUniforms::build (gpu.rs:147-211)."""
    cfg = _lib.RenderConfig(width, height, mode, shadow_mode, slice_mode, prophecy_delta)
    dyn = _lib.FrameDynamics()
    keep = []
    if frontier is not None:
        dyn.has_frontier = 1
        for k in range(4):
            dyn.frontier_origin[k] = frontier[0][k]
        dyn.frontier_tau = frontier[1]
    dyn.frontier_lag = frontier_lag
    if flashes:
        arr = (_lib.Flash * len(flashes))()
        for i, (at, w, inten, col) in enumerate(flashes):
            for k in range(4):
                arr[i].at[k] = at[k]
            arr[i].width, arr[i].intensity = w, inten
            for k in range(3):
                arr[i].color[k] = col[k]
        dyn.flashes = arr
        dyn.n_flashes = len(flashes)
        keep.append(arr)
    if remote_origins:
        ro = (C.c_float * (4 * len(remote_origins)))(*[float(v) for o in remote_origins for v in o])
        dyn.remote_origins = C.cast(ro, C.POINTER(C.c_float))
        dyn.n_remote = len(remote_origins)
        keep.append(ro)
    u = GpuUniforms()
    _check(_lib.lib().sr_uniforms_build(C.byref(cam), C.byref(cfg), C.byref(dyn), num_nodes,
                                        (C.c_float * 4)(*light_pos), num_stars, C.byref(u)), what="uniforms_build")
    return u


def observers(seed: int, n: int):
    arr = (_lib.ObserverDraw * n)()
    _check(_lib.lib().sr_observers_synth(seed, n, arr), what="observers")
    return [dict(width=o.width, height=o.height, slice_mode=o.slice_mode, pos=tuple(o.pos[:4]),
                 rapidity=tuple(o.rapidity[:3])) for o in arr]


def tables() -> np.ndarray:
    out = np.zeros(4096 + 14 * 7, np.uint32)
    _check(_lib.lib().sr_tables_build(out.ctypes.data_as(C.POINTER(C.c_uint32))), what="tables")
    return out


def cam64(event, rapidity=(0.0, 0.0, 0.0), yaw=0.0, pitch=0.0, roll=0.0) -> CameraF64:
    c = CameraF64()
    for k in range(4):
        c.event[k] = event[k]
    for k in range(3):
        c.rapidity[k] = rapidity[k]
    c.yaw, c.pitch, c.roll = yaw, pitch, roll
    return c


@dataclass
class Frame:
    rgb: np.ndarray
    hit_id: np.ndarray | None = None
    lam: np.ndarray | None = None
    tau: np.ndarray | None = None
    hdr: np.ndarray | None = None
    timings: _lib.Timings | None = None


def top_tree(boxes, roots, weights, base: int, depths=None):
    """sr_top_tree (bvh4d.rs:593-644, host): the n - 1 nodes over n subtrees and the tree's depth."""
    b = np.ascontiguousarray(boxes, np.float32)
    r = np.ascontiguousarray(roots, np.uint32)
    w = np.ascontiguousarray(weights, np.float32)
    d = None if depths is None else np.ascontiguousarray(depths, np.uint32)
    out = np.zeros(len(r) - 1, NODE_DTYPE)
    depth = C.c_uint32()
    _check(_lib.lib().sr_top_tree(b.ctypes.data, r.ctypes.data, w.ctypes.data, None if d is None else d.ctypes.data,
                                  len(r), base, out.ctypes.data, C.byref(depth)), what="top_tree")
    return out, depth.value


@dataclass
class TubeData:
    """One worldtube (SrTube): a mesh in its body frame swept along worldline samples."""
    vertices: np.ndarray              # (n, 3) float32
    triangles: np.ndarray             # TRI_DTYPE
    samples: np.ndarray               # SAMPLE_DTYPE
    material: int
    decided: np.ndarray | None = None  # per-sample causal decision stamps, or None (static)

    def struct(self):
        keep = [np.ascontiguousarray(self.vertices, np.float32), np.ascontiguousarray(self.triangles, TRI_DTYPE),
                np.ascontiguousarray(self.samples, SAMPLE_DTYPE)]
        t = _lib.Tube()
        t.vertices, t.triangles, t.samples = (a.ctypes.data for a in keep)
        t.num_vertices = len(keep[0])
        t.num_triangles = len(keep[1])
        t.num_samples = len(keep[2])
        t.material = self.material
        if self.decided is not None:
            d = np.ascontiguousarray(self.decided, np.float32)
            assert len(d) == len(keep[2])
            keep.append(d)
            t.decided_at = d.ctypes.data
        return t, keep


def _part(part) -> "_lib.ArenaPart":
    kind, player, pid = part
    return _lib.ArenaPart(kind, player, pid)


class Engine:
    """GpuRenderer over the C ABI: one CUDA context, scenes uploaded once, frames rendered on demand."""

    def __init__(self, device: int = 0):
        L = _lib.lib()
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = L.sr_create(device, C.byref(h), err, 512)
        if st != _lib.SR_OK:
            raise SrError(st, err.value.decode())
        self.h = h
        self.L = L
        self.scenes = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.sr_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def adapter_name(self) -> str:
        buf = C.create_string_buffer(256)
        _check(self.L.sr_adapter_name(self.h, buf, 256), self.h, "adapter_name")
        return buf.value.decode()

    def set_stream(self, stream_ptr: int | None):
        _check(self.L.sr_set_stream(self.h, stream_ptr), self.h, "set_stream")

    def synchronize(self):
        _check(self.L.sr_synchronize(self.h), self.h, "synchronize")

    def upload(self, idx: int, scene) -> None:
        d, keep = scene.desc()
        _check(self.L.sr_upload_scene(self.h, idx, C.byref(d)), self.h, "upload_scene")
        self.scenes[idx] = scene

    def build(self, idx: int, boxes: np.ndarray, geoms: np.ndarray, attrs: np.ndarray, materials: np.ndarray,
              stars: np.ndarray | None = None, num_stars: int = 0, light_pos=(0.0, 0.0, 50.0, 0.0), anchor=None) -> None:
        """sr_build_scene: the tree and leaf order built on the device from simplices in build order."""
        keep = [np.ascontiguousarray(boxes, np.float32), np.ascontiguousarray(geoms), np.ascontiguousarray(attrs),
                np.ascontiguousarray(materials)]
        d = _lib.BuildDesc()
        d.boxes, d.geoms, d.attrs, d.materials = (a.ctypes.data for a in keep)
        d.num_prims = len(geoms)
        d.num_materials = len(materials)
        if num_stars:
            st = np.ascontiguousarray(stars, np.float32)
            keep.append(st)
            d.stars = st.ctypes.data
            d.num_star_vec4 = st.size // 4
            d.num_stars = num_stars
        for k in range(4):
            d.light_pos[k] = light_pos[k]
        if anchor is not None:
            an = np.asarray(anchor, np.float64)
            keep.append(an)
            d.anchor = an.ctypes.data
        _check(self.L.sr_build_scene(self.h, idx, C.byref(d)), self.h, "build_scene")
        self.scenes[idx] = keep

    def build_tubes(self, idx: int, scene: "SynthScene") -> None:
        """sr_build_scene_tubes: the synthetic scene's worldtubes extruded, built and packed on the device."""
        tp = C.c_void_p()
        nt = C.c_uint32()
        _check(_lib.lib().sr_scene_tubes(scene.h, C.byref(tp), C.byref(nt)), what="scene_tubes")
        sd = scene._desc  # the scene's own arrays: materials, stars, light and anchor
        d = _lib.BuildDesc()
        d.materials = sd.materials
        d.num_materials = sd.num_materials
        d.stars = sd.stars
        d.num_star_vec4 = sd.num_star_vec4
        d.num_stars = sd.num_stars
        for k in range(4):
            d.light_pos[k] = sd.light_pos[k]
        d.anchor = sd.anchor
        _check(self.L.sr_build_scene_tubes(self.h, idx, tp, nt.value, C.byref(d)), self.h, "build_scene_tubes")
        self.scenes[idx] = scene

    # ---- the scene cache over a device arena (SceneCache, dynamic/scene_cache.rs) ----
    def arena_begin(self, idx: int) -> None:
        _check(self.L.sr_arena_begin(self.h, idx), self.h, "arena_begin")

    def arena_tube(self, idx: int, part, tube: TubeData) -> None:
        """SceneCache::tube; part = (kind, player, id) with kind 0 body, 1 hull, 2 pulse."""
        t, keep = tube.struct()
        _check(self.L.sr_arena_tube(self.h, idx, _part(part), C.byref(t)), self.h, "arena_tube")

    def arena_piece(self, idx: int, part, index: int, key, boxes, geoms, attrs) -> bool:
        """SceneCache::piece: returns whether the chunk was reused (else its simplices are installed)."""
        k = np.ascontiguousarray(key, np.uint32)
        reused = C.c_int32()
        _check(self.L.sr_arena_reuse(self.h, idx, _part(part), index, k.ctypes.data, len(k), C.byref(reused)),
               self.h, "arena_reuse")
        if not reused.value:
            b = np.ascontiguousarray(boxes, np.float32)
            g = np.ascontiguousarray(geoms, GEOM_DTYPE)
            a = np.ascontiguousarray(attrs, ATTR_DTYPE)
            _check(self.L.sr_arena_install(self.h, idx, _part(part), index, b.ctypes.data, g.ctypes.data,
                                           a.ctypes.data, len(g)), self.h, "arena_install")
        return bool(reused.value)

    def arena_finish(self, idx: int, rest: "SynthScene", boxes=None, geoms=None, attrs=None) -> dict:
        """SceneCache::finish with the volatile simplices (build order, may be None); materials, stars,
        light and anchor from `rest`. Returns the snapshot's CacheStats."""
        sd = rest._desc
        d = _lib.BuildDesc()
        keep = []
        if geoms is not None and len(geoms):
            keep = [np.ascontiguousarray(boxes, np.float32), np.ascontiguousarray(geoms, GEOM_DTYPE),
                    np.ascontiguousarray(attrs, ATTR_DTYPE)]
            d.boxes, d.geoms, d.attrs = (a.ctypes.data for a in keep)
            d.num_prims = len(keep[1])
        d.materials = sd.materials
        d.num_materials = sd.num_materials
        d.stars = sd.stars
        d.num_star_vec4 = sd.num_star_vec4
        d.num_stars = sd.num_stars
        for k in range(4):
            d.light_pos[k] = sd.light_pos[k]
        d.anchor = sd.anchor
        st = _lib.ArenaStats()
        _check(self.L.sr_arena_finish(self.h, idx, C.byref(d), C.byref(st)), self.h, "arena_finish")
        self.scenes[idx] = rest
        return {k: getattr(st, k) for k, _ in _lib.ArenaStats._fields_}

    def records(self, idx: int):
        """The device scene's hot and cold records (leaf order)."""
        n = self.stats(idx).num_prims
        g = np.zeros(n, GEOM_DTYPE)
        a = np.zeros(n, ATTR_DTYPE)
        _check(self.L.sr_scene_records(self.h, idx, g.ctypes.data, a.ctypes.data, n), self.h, "scene_records")
        return g, a

    def tree(self, idx: int):
        """The device scene's node array and leaf order (leaf slot -> build index)."""
        nn = C.c_uint32()
        _check(self.L.sr_scene_tree(self.h, idx, None, 0, None, 0, C.byref(nn)), self.h, "scene_tree")
        nodes = np.zeros(nn.value, NODE_DTYPE)
        n = self.stats(idx).num_prims
        order = np.zeros(n, np.uint32)
        _check(self.L.sr_scene_tree(self.h, idx, nodes.ctypes.data, nn.value, order.ctypes.data, n, C.byref(nn)),
               self.h, "scene_tree")
        return nodes, order

    def update(self, idx: int, scene, node_ranges=(), prim_ranges=()) -> None:
        d, keep = scene.desc()
        nr = (_lib.Range * max(1, len(node_ranges)))(*[_lib.Range(a, b) for a, b in node_ranges])
        pr = (_lib.Range * max(1, len(prim_ranges)))(*[_lib.Range(a, b) for a, b in prim_ranges])
        _check(self.L.sr_update_scene(self.h, idx, C.byref(d), nr, len(node_ranges), pr, len(prim_ranges)),
               self.h, "update_scene")
        self.scenes[idx] = scene

    def set_layout(self, idx: int, layout: int) -> None:
        """sr_set_layout: SR_LAYOUT_AUTO / OCTANT / COMPACT for the scene at `idx` (rebuilt now if present)."""
        _check(self.L.sr_set_layout(self.h, idx, layout), self.h, "set_layout")

    def stats(self, idx: int) -> _lib.SceneStats:
        s = _lib.SceneStats()
        _check(self.L.sr_scene_stats(self.h, idx, C.byref(s)), self.h, "scene_stats")
        return s

    def render(self, idx: int, u: GpuUniforms, path: int = SR_PATH_FAST, aux: bool = False, hdr: bool = False,
               timing: bool = False, cam: CameraF64 | None = None, count: bool = False,
               star_brute: bool = False) -> Frame:
        n = u.size[0] * u.size[1]
        fr = Frame(rgb=np.zeros(n, np.uint32))
        out = _lib.Outputs()
        out.rgb = fr.rgb.ctypes.data
        if aux:
            fr.hit_id = np.zeros(n, np.uint32)
            fr.lam = np.zeros(n, np.float32)
            fr.tau = np.zeros(n, np.float32)
            out.hit_id, out.lambda_, out.tau = fr.hit_id.ctypes.data, fr.lam.ctypes.data, fr.tau.ctypes.data
        if hdr:
            fr.hdr = np.zeros((n, 4), np.float32)
            out.hdr = fr.hdr.ctypes.data
        flags = (SR_FLAG_TIMING if timing else 0) | (_lib.SR_FLAG_COUNT_WORK if count else 0)
        flags |= _lib.SR_FLAG_STAR_BRUTE if star_brute else 0
        opts = _lib.RenderOpts(path, flags, C.pointer(cam) if cam is not None else None)
        t = _lib.Timings()
        _check(self.L.sr_render_ex(self.h, idx, C.byref(u), C.byref(opts), C.byref(out), C.byref(t)), self.h,
               "render")
        fr.timings = t
        return fr

    def render_into(self, idx: int, u: GpuUniforms, rgb_ptr: int, path: int = SR_PATH_FAST, device_output=True,
                    timing: bool = False, cam: CameraF64 | None = None, timings: _lib.Timings | None = None) -> None:
        """Render into a raw pointer (device memory with device_output, else host)."""
        out = _lib.Outputs()
        out.rgb = rgb_ptr
        flags = (SR_FLAG_DEVICE_OUTPUT if device_output else 0) | (SR_FLAG_TIMING if timing else 0)
        opts = _lib.RenderOpts(path, flags, C.pointer(cam) if cam is not None else None)
        _check(self.L.sr_render_ex(self.h, idx, C.byref(u), C.byref(opts), C.byref(out),
                                   C.byref(timings) if timings is not None else None), self.h, "render")

    def render_host(self, idx: int, u: GpuUniforms, fb: np.ndarray) -> _lib.Timings:
        """sr_render: the drop-in GpuRenderer::render (host framebuffer, blocking)."""
        t = _lib.Timings()
        _check(self.L.sr_render(self.h, idx, C.byref(u), fb.ctypes.data, fb.size, C.byref(t)), self.h, "render")
        return t

    def render_batch(self, idx: int, us: list, rgb_ptr: int, rgb_len: int, cams: list | None = None,
                     device_output: bool = True, timing: bool = False, phases: bool = False,
                     count: bool = False, star_brute: bool = False, async_output: bool = False) -> _lib.Timings:
        """Renders observers `us` into `rgb_ptr` (concatenated frames). `timing` returns the batch's
        device time; `phases` adds per-phase times, `count` the traversal work (both run the launch
        sequence outside its CUDA graph). `async_output` (host framebuffer, pinned for overlap):
        return once queued; the frames are there after `synchronize()`."""
        n = len(us)
        ua = (GpuUniforms * n)(*us)
        ca = (CameraF64 * n)(*cams) if cams else None
        t = _lib.Timings()
        flags = SR_FLAG_DEVICE_OUTPUT if device_output else 0
        flags |= (_lib.SR_FLAG_TIMING if phases else 0) | (_lib.SR_FLAG_COUNT_WORK if count else 0)
        flags |= _lib.SR_FLAG_STAR_BRUTE if star_brute else 0
        flags |= _lib.SR_FLAG_ASYNC_OUTPUT if async_output else 0
        timing = timing or phases or count
        _check(self.L.sr_render_batch(self.h, idx, ua, ca, n, rgb_ptr, rgb_len, flags,
                                      C.byref(t) if timing else None), self.h, "render_batch")
        return t

    def adjoint(self, idx: int, u: GpuUniforms, cam: CameraF64, target_hdr_ptr: int, level: int = 0,
                frozen: bool = False, rows: tuple[int, int] | None = None) -> _lib.AdjointResult:
        """Loss sum((P(HDR) - P(target))^2) of the observer `cam` (P: `level` 2x2 box halvings) and
        its gradient with respect to (rapidity x, y, z, event t, x, y, z); `target_hdr_ptr`: device,
        width*height*4 floats. `frozen`: the loss only, under the previous call's discrete outcomes.
        `rows`: only rows [begin, end) of the loss level (sr_adjoint_rows)."""
        r = _lib.AdjointResult()
        flags = _lib.SR_ADJ_FROZEN if frozen else 0
        if rows is None:
            st = self.L.sr_adjoint(self.h, idx, C.byref(u), C.byref(cam), target_hdr_ptr, level, flags, C.byref(r))
        else:
            st = self.L.sr_adjoint_rows(self.h, idx, C.byref(u), C.byref(cam), target_hdr_ptr, level, flags, rows[0],
                                        rows[1], C.byref(r))
        _check(st, self.h, "adjoint")
        return r

    def trace_rays(self, idx: int, rays) -> np.ndarray:
        """sr_trace_rays: Bvh4D::trace and interpolate_hit of rays (n x 10: origin t, x, y, z as
        doubles, direction, t_min, t_max) on the device. Returns a structured array of SrRayHit."""
        r = np.atleast_2d(np.asarray(rays, np.float64))
        n = len(r)
        arr = (_lib.Ray * max(n, 1))()
        for i in range(n):
            arr[i].origin[:] = list(r[i, 0:4])
            arr[i].dir[:] = list(np.float32(r[i, 4:8]))
            arr[i].t_min, arr[i].t_max = float(np.float32(r[i, 8])), float(np.float32(r[i, 9]))
        out = (_lib.RayHit * max(n, 1))()
        _check(self.L.sr_trace_rays(self.h, idx, arr, n, out), self.h, "trace_rays")
        return np.ctypeslib.as_array(out)[:n].copy()

    def tuning(self, idx: int) -> _lib.Tuning:
        t = _lib.Tuning()
        _check(self.L.sr_get_tuning(self.h, idx, C.byref(t)), self.h, "get_tuning")
        return t

    def set_tuning(self, idx: int, t: _lib.Tuning):
        _check(self.L.sr_set_tuning(self.h, idx, C.byref(t)), self.h, "set_tuning")

    def autotune(self, idx: int, u: GpuUniforms, n: int = 3):
        best = _lib.Tuning()
        ms = C.c_float()
        _check(self.L.sr_autotune(self.h, idx, C.byref(u), n, C.byref(best), C.byref(ms)), self.h, "autotune")
        return best, ms.value
