#!/usr/bin/env python
"""Headline benchmark: primary rays per second on the 7.9M-tetrahedron 1280x800 scene.

Workload: 64 accelerated icospheres (subdivision 2) on Fermi-Walker worldlines, 128 time steps,
~7.9M tetrahedra; observers at t = 0 at the origin with rapidities |phi| <= 2; 1280x800; past
light cone; Lorentz-invariant null shadows from a point light at (0, 50, 0); FP32 traversal.
Synthetic, seeded (the reference ships no scenes for these configurations).

One step renders a batch of B observers (B frames of 1,024,000 rays each) through the batched
fast path with the FP64 camera (tetrad and event built in double on the GPU, rebased to the scene
anchor). `value` is Mrays/s over all ranks (weak scaling: every rank renders its own batch of
observers, no data-path collective). The same line carries:

  plain        the plain single-frame path on the same observers (batched over plain: the metric's
               "batched vs plain");
  parity       observer 0's frame against the all-FP64 oracle (scene built and rendered in double):
               hit-id agreement (the metric's "hit-ID match % vs FP64"), lambda / tau / RGB errors;
  e2e          the same batches through the C ABI with host buffers;
  value_fresh  every step a new seeded set of observers, L2 flushed before each step;
  traversal_per_ray  the same batches with each ray walking the tree alone (no warp packets);
  config4      64 observers of mixed resolution and slice mode over the 147k-tet cube scene in one
               batch, against looping the plain path;
  config5      the image-loss gradient of one 1280x800 observer over 100k stars;
  cpu_baseline the oracle (C++ restatement of the reference's CPU renderer) on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

`--impl reference` times the reference's CPU renderer (its C++ restatement in oracle/: the Rust
renderer cannot be built here) on the host cores, on the same scene (built by the oracle) and the
same observers, each on a sample of every 8th row.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 1280, 800
RAYS_PER_FRAME = W * H
METRIC = "Mrays/s on 1 B200, 1280×800 8M-tet scene, batched vs plain; hit-ID match % vs FP64"
UNIT = "Mrays/s"
ROW_STRIDE = 8  # the CPU arms render every 8th row of each frame


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--batch", type=int, default=8, help="observers (1280x800 frames) per step per GPU")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the FP64-oracle parity block")
    ap.add_argument("--no-extra", action="store_true", help="skip the config4 / config5 / fresh-observer legs")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch parameters")
    ap.add_argument("--no-roof", action="store_true",
                    help="skip the coherent-ray roof (24 extra batches; for profiler launch lists)")
    ap.add_argument("--bodies", type=int, default=64,
                    help="icospheres in the scene (64 is the workload; fewer only for small profiling captures)")
    ap.add_argument("--workload", choices=["config2", "config4", "config5", "tunings"], default="config2",
                    help="config2: the headline (8 observers of the 7.9M-tet scene per step, with the config4 and "
                         "config5 legs as extra keys); config4 / config5 alone: see run_config4 / run_config5")
    return ap.parse_args()


def load_shard():
    """specrel_b200/shard.py (numpy only) loaded by path, so that the reference arm maps no engine code."""
    spec = importlib.util.spec_from_file_location("sr_shard", os.path.join(ROOT, "specrel_b200", "shard.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_config(args, world):
    """The `config` of both arms (identical, so the two lines describe the same workload)."""
    return {"workload": "64 accelerated icospheres (subdiv 2), 128 steps, 7,864,320 tets, 1280x800, past light "
                        "cone, Lorentz-invariant null shadows, light (0,50,0), FP32 traversal + FP64 camera",
            "observers_per_step_per_gpu": args.batch, "seed": args.seed, "bodies": args.bodies,
            "l2": "inputs larger than L2 (the scene is >2.6 GB on the device against a 126 MB L2); value_fresh "
                  "also renders new observers every step with L2 flushed before each",
            "parallelism": f"replicas x{world}, observers sharded"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def oracle_row_config(O, stride=ROW_STRIDE):
    """Every `stride`-th row of the 1280x800 frame (1280 x 800/stride rays), shadows on."""
    return O.make_config(W, H // stride, 0, 1, 0, full_height=H, row_stride=stride, row_offset=stride // 2)


def cpu_baseline(packed, rapidities):
    """The reference CPU renderer (oracle/: the C++ restatement of renderer.rs, f32, rows over all
    host threads, serial bloom) on a bounded sample of the same step: each observer's every 8th row
    (1280 x 100 rays per observer), one warm-up then the median of 3 passes."""
    from oracle import oracle as O
    sc = O.Scene.from_packed(packed.nodes, packed.geoms, packed.attrs, packed.materials, packed.stars,
                             packed.num_stars, packed.light_pos)
    cams = [O.make_camera(rapidity=r) for r in rapidities]
    cfg = oracle_row_config(O)
    threads = os.cpu_count() or 1
    for c in cams:
        O.render(sc, c, cfg, threads=threads, aux=False)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        for c in cams:
            O.render(sc, c, cfg, threads=threads, aux=False)
        ts.append(time.perf_counter() - t0)
    t = float(np.median(ts))
    rays = W * (H // ROW_STRIDE) * len(cams)
    return {"value": rays / t / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"rows {ROW_STRIDE // 2}::{ROW_STRIDE} of each of the step's {len(cams)} observers' frames "
                      f"({rays} rays, shadows on, bloom on the sample), oracle C++ f32 restatement of render_frame, "
                      f"median of 3 after a warm-up; {t * 1e3:.1f} ms per pass"}


def run_reference(args, rank, world):
    """The reference arm. The reference's CPU renderer is Rust (renderer.rs:327-412) and cannot be
    built here (no cargo / rustc), so its C++ restatement in oracle/ is timed on all host cores. The
    scene is built by the oracle itself (the same arrays as the engine's scene builder produces),
    and each step renders the engine arm's observers, each on every 8th row of its frame."""
    if rank != 0:
        return
    from oracle import oracle as O
    shard = load_shard()
    t0 = time.time()
    sc = O.Scene(O.synth_params(2, args.seed, n_bodies=args.bodies))
    build_s = time.time() - t0
    raps = shard.observer_rapidities(args.seed, 0, args.batch, tuple(sc.info.cam_rapidity))
    cams = [O.make_camera(rapidity=r) for r in raps]
    cfg = oracle_row_config(O)
    threads = os.cpu_count() or 1

    def step():
        for c in cams:
            O.render(sc, c, cfg, threads=threads, aux=False)

    for _ in range(args.warmup):
        step()
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        ts.append(time.perf_counter() - t0)
    t = float(np.mean(ts))
    rays = W * (H // ROW_STRIDE) * len(cams)
    v = rays / t / 1e6
    sample = (f"each step: rows {ROW_STRIDE // 2}::{ROW_STRIDE} of each of the {len(cams)} observers' 1280x800 frames "
              f"({rays} rays), all {threads} host threads; the Rust renderer is not buildable here (no cargo/rustc), "
              "so the oracle's C++ restatement of render_frame is timed")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "impl": "reference",
            "data": "synthetic (seeded accelerated-icosphere scene, built by the oracle)",
            "config": workload_config(args, world), "rays_per_step": rays, "scene_build_s": round(build_s, 2),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def parity_fp64(args, eng, u0, cam0, rap0):
    """Observer 0's frame on the fast path with the FP64 camera (the measured configuration)
    against the all-FP64 oracle: the scene built and rendered in double, the whole 1280x800 frame
    (bloom included), on the host cores."""
    import specrel_b200 as sr
    from oracle import oracle as O
    t0 = time.time()
    s64 = O.Scene(O.synth_params(2, args.seed, n_bodies=args.bodies), fp64=True)
    ref = O.render(s64, O.make_camera(rapidity=rap0), O.make_config(W, H, 0, 1, 0), threads=os.cpu_count() or 1)
    del s64
    fr = eng.render(0, u0, path=sr.SR_PATH_FAST, aux=True, cam=cam0)
    miss = 0xFFFFFFFF
    gid, oid = fr.hit_id.astype(np.uint32), ref.orig.astype(np.uint32)
    same = gid == oid
    hit = same & (gid != miss)
    lam = np.abs(fr.lam[hit].astype(np.float64) - ref.lam[hit]) / np.abs(ref.lam[hit])
    tau = np.abs(fr.tau[hit].astype(np.float64) - ref.tau[hit]) / np.maximum(np.abs(ref.tau[hit]), 1.0)

    def ch(x):
        x = x.astype(np.uint32)
        return np.stack([(x >> 16) & 255, (x >> 8) & 255, x & 255], -1).astype(np.int32)

    d = np.abs(ch(fr.rgb) - ch(ref.rgb)).max(-1)
    return {"reference": "all-FP64 oracle (scene built and rendered in double), observer 0, whole 1280x800 frame",
            "pixels": int(same.size), "hit_id_match_pct": float(same.mean() * 100.0),
            "hit_id_mismatches": int((~same).sum()),
            "lambda_rel_max": float(lam.max()), "lambda_rel_median": float(np.median(lam)),
            "tau_rel_max": float(tau.max()), "tau_rel_median": float(np.median(tau)),
            "rgb8_max_abs": int(d.max()), "rgb8_max_abs_on_agreeing_hits": int(d[same].max()),
            "rgb8_frac_gt1": float((d > 1).mean()), "seconds": round(time.time() - t0, 1)}


def config4_measure(args, rank, world, local, dist, stream, eng, idx):
    """The cube scene (64 inertial unit cubes, 147k tets) seen by 64 observers in one batch:
    resolutions drawn from {320x200, 640x400, 1280x800, 1920x1200}, events t in [-50, 0] with
    |x| <= 30, rapidities |phi| <= 3, half past light cone and half God's-eye slice. One step = the
    whole batch through the batched fast path with FP64 cameras (one captured graph); `plain` loops
    the plain single-frame path over the same observers. Observers are sharded over ranks."""
    import torch
    import specrel_b200 as sr
    from specrel_b200 import shard
    scene = sr.synth_scene(1, args.seed)
    eng.upload(idx, scene)
    draws = [o for i, o in enumerate(sr.observers(args.seed, 64)) if i % world == rank]
    us, cams = [], []
    for o in draws:
        c = sr.camera(tuple(o["pos"]), 90.0, rapidity=o["rapidity"])
        us.append(sr.uniforms(c, o["width"], o["height"], 0, 1 if o["slice_mode"] == 0 else 2, o["slice_mode"],
                              num_nodes=scene.num_nodes, light_pos=scene.light_pos))
        cams.append(sr.cam64(o["pos"], o["rapidity"]))
    rays = sum(u.size[0] * u.size[1] for u in us)
    out = torch.empty(max(rays, 1), dtype=torch.int32, device=f"cuda:{local}")
    ptr = out.data_ptr()

    def timed(fn, k):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return shard.max_over_ranks(e0.elapsed_time(e1) / k, dist, f"cuda:{local}")

    def batch_step():
        eng.render_batch(idx, us, ptr, rays, cams=cams, device_output=True)

    def plain_step():
        off = 0
        for u in us:
            eng.render_into(idx, u, ptr + 4 * off, path=sr.SR_PATH_PLAIN)
            off += u.size[0] * u.size[1]

    with torch.cuda.stream(stream):
        if not args.no_autotune:
            eng.autotune(idx, us[0], 8)
        ms = timed(batch_step, args.steps)
        plain_ms = timed(plain_step, max(2, args.steps // 2))
        ph = eng.render_batch(idx, us, ptr, rays, cams=cams, device_output=True, phases=True)
    total = rays
    if dist is not None:
        t = torch.tensor([rays], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t)
        total = int(t.item())
    sizes = {}
    for o in draws:
        key = f"{o['width']}x{o['height']}"
        sizes[key] = sizes.get(key, 0) + 1
    value = total / (ms / 1e3) / 1e6
    plain_value = total / (plain_ms / 1e3) / 1e6
    tuning = eng.tuning(idx)
    res = {"metric": "Mrays/s, 64 observers of the 147k-tet cube scene in one batch; primary rays",
           "value": value, "unit": UNIT, "ms_per_step": ms, "rays_per_step": total,
           "workload": f"{scene.num_prims} tets, 64 observers (sizes {sizes}), past light cone and God's-eye "
                       "slice 50/50, FP64 cameras; scene L2-resident",
           "plain": {"value": plain_value, "unit": UNIT, "ms_per_step": plain_ms},
           "speedup_batched_over_plain": value / plain_value,
           "phases_ms": {"trace": ph.trace_ms, "shade": ph.shade_ms, "stars": ph.stars_ms, "bloom": ph.bloom_ms},
           "tuning": {k: getattr(tuning, k)
                      for k, _ in tuning._fields_}}
    del out
    return res


def config5_measure(args, local, stream, eng, idx):
    """100k inertial stars on a sphere of radius 1e3 over the cube scene, 1280x800, target rendered
    at rapidity (0.8, -0.3, 0.5). Times, with CUDA events on the engine's stream: one forward frame
    on the fast path (FP64 camera, binned stars) and one loss-and-gradient evaluation (sr_adjoint:
    the forward frame recomputed, then the 7-vector of rapidity and event derivatives in f32 with
    f64 sums) at loss level 0 (full resolution) and level 3, from rapidity 0."""
    import torch
    import specrel_b200 as sr
    scene = sr.synth_scene(5, args.seed)
    eng.upload(idx, scene)
    star = (0.8, -0.3, 0.5)
    u = sr.uniforms(sr.camera(), W, H, 0, 1, 0, num_nodes=scene.num_nodes, num_stars=scene.num_stars,
                    light_pos=scene.light_pos)
    ev = (0.0, 0.0, 0.0, 0.0)
    out = torch.empty(W * H, dtype=torch.int32, device=f"cuda:{local}")
    with torch.cuda.stream(stream):
        tgt = eng.render(idx, u, path=sr.SR_PATH_FAST, hdr=True, cam=sr.cam64(ev, star)).hdr
        tdev = torch.tensor(tgt, device=f"cuda:{local}").contiguous()
        cam0 = sr.cam64(ev, (0.0, 0.0, 0.0))

        def timed(fn, k):
            for _ in range(max(1, args.warmup)):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / k

        fwd = timed(lambda: eng.render_into(idx, u, out.data_ptr(), path=sr.SR_PATH_FAST, cam=cam0), args.steps)
        g0 = timed(lambda: eng.adjoint(idx, u, cam0, tdev.data_ptr(), 0), args.steps)
        g3 = timed(lambda: eng.adjoint(idx, u, cam0, tdev.data_ptr(), 3), args.steps)
        r = eng.adjoint(idx, u, cam0, tdev.data_ptr(), 0)
    res = {"metric": "ms per image-loss gradient, 100k stars over the cube scene, 1280x800",
           "value": g0, "unit": "ms", "higher_is_better": False,
           "workload": f"{scene.num_prims} tets, {scene.num_stars} stars, 1280x800, target at rapidity "
                       "(0.8, -0.3, 0.5), gradient at rapidity 0",
           "forward_frame_ms": fwd, "gradient_level3_ms": g3,
           "gradient": {"loss": r.loss, "grad": list(r.grad), "star_terms": r.star_terms,
                        "primal_mismatch": r.primal_mismatch}}
    del tdev, out
    return res


def coherent_roof(sr, eng, scene, ptr, B, seed, work, trace_ms):
    """The trace kernel's ceiling on this GPU, measured in this run: batches in which every pixel of
    a frame traces that frame's centre ray (half_wh = 0), so the 32 lanes of a warp take the same
    nodes and tests in step, no lane idles, and every load after a warp's first is an L1 hit. The
    kernel's time on such batches, least squares (non-negative) over per-launch, per-node-visit,
    per-tetrahedron-test and per-shadow-ray costs, gives the time the same kernel would take on the
    real batch's work if its rays were coherent: the roof. frac = roof time / measured time.
    Centre rays vary by observer rapidity, yaw and pitch, slice (past cone, God's-eye, future
    cone) and shadows on / off, so the work mix varies across the fitted batches.
    Only for scenes without stars (the binned-star set-up divides by the pixel pitch)."""
    from scipy.optimize import nnls
    rng = np.random.default_rng(seed * 31 + 7)
    X, y = [], []
    for slice_mode in (0, 1, 2):
        for shadow in (1, 0):
            for _ in range(4):
                while True:
                    r = rng.uniform(-1.0, 1.0, 3)
                    if r @ r < 1.0:
                        break
                r = tuple(float(v) for v in 2.0 * r)
                yaw, pitch = float(rng.uniform(-0.5, 0.5)), float(rng.uniform(-0.35, 0.35))
                u = sr.uniforms(sr.camera(rapidity=r), W, H, 0, shadow, slice_mode, num_nodes=scene.num_nodes,
                                light_pos=scene.light_pos)
                u.half_wh[0] = 0.0
                u.half_wh[1] = 0.0
                c = sr.cam64((0.0, 0.0, 0.0, 0.0), r, yaw, pitch)
                ub, cb = [u] * B, [c] * B
                eng.render_batch(0, ub, ptr, B * RAYS_PER_FRAME, cams=cb, device_output=True)
                ts = [eng.render_batch(0, ub, ptr, B * RAYS_PER_FRAME, cams=cb, device_output=True,
                                       phases=True).trace_ms for _ in range(3)]
                t = eng.render_batch(0, ub, ptr, B * RAYS_PER_FRAME, cams=cb, device_output=True, count=True)
                X.append([1.0, float(t.nodes_visited + t.shadow_nodes_visited),
                          float(t.tets_tested + t.shadow_tets_tested), float(t.shadow_rays)])
                y.append(float(np.median(ts)))
    X, y = np.array(X), np.array(y)
    scale = np.maximum(X.max(axis=0), 1.0)
    coef, _ = nnls(X / scale, y)
    coef = coef / scale
    fit = X @ coef
    real = np.array([1.0, work[0] + work[3], work[2] + work[5], work[6]])
    roof_ms = float(real @ coef)
    rays = B * RAYS_PER_FRAME
    return {
        "achieved": rays / (trace_ms / 1e3) / 1e6, "peak": rays / (roof_ms / 1e3) / 1e6, "unit": "Mrays/s",
        "frac": roof_ms / trace_ms, "roof_ms_per_launch": roof_ms,
        "peak_kind": "measured in this run: the same kernel on warp-coherent batches (every pixel of a frame on "
                     "its centre ray), its per-launch, per-node-visit, per-test and per-shadow-ray costs fitted "
                     "and applied to this batch's counted work",
        "coherent_fit": {"batches": int(len(y)), "ms_per_launch": float(coef[0]),
                         "ns_per_node_visit": float(coef[1] * 1e6), "ns_per_tet_test": float(coef[2] * 1e6),
                         "ns_per_shadow_ray": float(coef[3] * 1e6),
                         "max_rel_residual": float(np.max(np.abs(fit - y) / y)),
                         "trace_ms_range": [float(y.min()), float(y.max())],
                         "node_visits_per_launch_range": [float(X[:, 1].min()), float(X[:, 1].max())],
                         "tet_tests_per_launch_range": [float(X[:, 2].min()), float(X[:, 2].max())]},
    }


def run_engine(args, rank, world, local):
    import torch
    import specrel_b200 as sr
    from specrel_b200 import shard
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ncpu = os.cpu_count() or 1
    t0 = time.time()
    scene = sr.synth_scene(2, args.seed, n_bodies=args.bodies, threads=max(1, ncpu // max(1, world)))
    build_s = time.time() - t0
    eng = sr.Engine(local)
    eng.upload(0, scene)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    B = args.batch
    raps = shard.observer_rapidities(args.seed, rank, B, scene.info.cam_rapidity)
    cams = [sr.camera(rapidity=r) for r in raps]
    us = [sr.uniforms(c, W, H, 0, 1, 0, num_nodes=scene.num_nodes, light_pos=scene.light_pos) for c in cams]
    c64 = [sr.cam64((0.0, 0.0, 0.0, 0.0), r) for r in raps]
    out = torch.empty(B * RAYS_PER_FRAME, dtype=torch.int32, device=f"cuda:{local}")
    ptr = out.data_ptr()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return shard.max_over_ranks(x, dist, f"cuda:{local}")

    extra = {}
    with torch.cuda.stream(stream):
        # Launch parameters for this scene, untimed.
        if not args.no_autotune:
            eng.autotune(0, us[0], B)

        def batch_step():
            eng.render_batch(0, us, ptr, B * RAYS_PER_FRAME, cams=c64, device_output=True)

        def plain_step():
            for i in range(B):
                eng.render_into(0, us[i], ptr + 4 * i * RAYS_PER_FRAME, path=sr.SR_PATH_PLAIN)

        for _ in range(args.warmup):
            batch_step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            torch.cuda.nvtx.range_push("timed")
            e0.record(stream)
            for _ in range(args.steps):
                batch_step()
            e1.record(stream)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        barrier()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        ms_max = max_over_ranks(ms)

        # The plain single-frame path on the same observers.
        for _ in range(max(1, args.warmup)):
            plain_step()
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        k_plain = max(2, args.steps // 2)
        for _ in range(k_plain):
            plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(e0.elapsed_time(e1) / k_plain)

        # End to end through the C ABI with host buffers: uniforms from pinned host memory in,
        # framebuffers out to pinned host memory, every step; each step's readback runs beside the
        # next step's render (SR_FLAG_ASYNC_OUTPUT), and the last one is waited for inside the
        # timed region.
        host = torch.empty(B * RAYS_PER_FRAME, dtype=torch.int32, pin_memory=True)
        hptr = host.data_ptr()
        for _ in range(max(1, args.warmup)):
            eng.render_batch(0, us, hptr, B * RAYS_PER_FRAME, cams=c64, device_output=False, async_output=True)
        eng.synchronize()
        barrier()
        torch.cuda.synchronize()
        t_e2e = time.perf_counter()
        e0.record(stream)
        for _ in range(args.steps):
            eng.render_batch(0, us, hptr, B * RAYS_PER_FRAME, cams=c64, device_output=False, async_output=True)
        eng.synchronize()
        e1.record(stream)
        torch.cuda.synchronize()
        wall_e2e = (time.perf_counter() - t_e2e) / args.steps * 1e3
        e2e_ms = max_over_ranks(max(e0.elapsed_time(e1) / args.steps, wall_e2e))

        # The compact node layout (one copy of the child boxes instead of 16 sign-octant copies) on
        # the same batches: what the octant copies cost in memory and buy in speed.
        # Every rank takes the leg or none does (the automatic layout depends on each GPU's free
        # memory, and the leg holds a collective).
        compact = None
        all_octant = max_over_ranks(0.0 if eng.stats(0).box_copies == 16 else 1.0) == 0.0
        if not args.no_extra and all_octant:
            eng.set_layout(0, sr._lib.SR_LAYOUT_COMPACT)
            compact_stats = eng.stats(0)
            for _ in range(max(1, args.warmup)):
                batch_step()
            torch.cuda.synchronize()
            barrier()
            e0.record(stream)
            for _ in range(args.steps):
                batch_step()
            e1.record(stream)
            torch.cuda.synchronize()
            compact_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
            eng.set_layout(0, sr._lib.SR_LAYOUT_AUTO)
            compact = (compact_stats, compact_ms)

        # The per-ray traversal (each ray walks the tree alone, SrTuning.packet = 0) on the same
        # batches, at its best measured launch shape: what the packet walk buys.
        per_ray_ms = None
        if not args.no_extra:
            keep = eng.tuning(0)
            t = eng.tuning(0)
            t.packet, t.block_threads, t.blocks_per_sm, t.stack_smem, t.top_levels = 0, 128, 11, 0, 0
            eng.set_tuning(0, t)
            for _ in range(max(1, args.warmup)):
                batch_step()
            torch.cuda.synchronize()
            barrier()
            e0.record(stream)
            for _ in range(args.steps):
                batch_step()
            e1.record(stream)
            torch.cuda.synchronize()
            per_ray_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
            eng.set_tuning(0, keep)

        # Fresh observers every step (new seeded rapidities, never rendered before), with L2 flushed
        # (a 256 MiB write) before each step; only the batches are inside the events.
        if not args.no_extra:
            flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
            fresh = []
            for k in range(args.steps):
                rk = shard.observer_rapidities(args.seed + 1000 + k, rank, B)
                fresh.append(([sr.uniforms(sr.camera(rapidity=r), W, H, 0, 1, 0, num_nodes=scene.num_nodes,
                                           light_pos=scene.light_pos) for r in rk],
                              [sr.cam64((0.0, 0.0, 0.0, 0.0), r) for r in rk]))
            barrier()
            torch.cuda.synchronize()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            for k, (fu, fc) in enumerate(fresh):
                flush.fill_(k & 255)
                evs[k][0].record(stream)
                eng.render_batch(0, fu, ptr, B * RAYS_PER_FRAME, cams=fc, device_output=True)
                evs[k][1].record(stream)
            torch.cuda.synchronize()
            fresh_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs) / args.steps)
            del flush

        # The dominant kernel (k_trace_lean: primary rays and the main light's shadow rays of all
        # B observers in one launch), timed with CUDA events the library records on the launching
        # stream around each phase of the same batch, then the traversal work of that batch
        # (counting variant).
        trace_ms, frame_ms, shade_ms, bloom_ms = [], [], [], []
        for _ in range(args.steps):
            t = eng.render_batch(0, us, ptr, B * RAYS_PER_FRAME, cams=c64, device_output=True, phases=True)
            trace_ms.append(t.trace_ms)
            shade_ms.append(t.shade_ms)
            bloom_ms.append(t.bloom_ms)
            frame_ms.append(t.kernel_ms)
        t = eng.render_batch(0, us, ptr, B * RAYS_PER_FRAME, cams=c64, device_output=True, count=True)
        work = np.array([t.nodes_visited, t.leaves_visited, t.tets_tested, t.shadow_nodes_visited,
                         t.shadow_leaves_visited, t.shadow_tets_tested, t.shadow_rays], dtype=np.float64)
        tuning = eng.tuning(0)
        stats = eng.stats(0)
        roof = None
        if scene.num_stars == 0 and not args.no_roof:
            roof = coherent_roof(sr, eng, scene, ptr, B, args.seed, work, float(np.median(trace_ms)))

        if not args.no_extra:
            extra["config4"] = config4_measure(args, rank, world, local, dist, stream, eng, 1)
            if rank == 0:
                extra["config5"] = config5_measure(args, local, stream, eng, 2)
        if rank == 0 and world == 1 and not args.no_parity:
            extra["parity"] = parity_fp64(args, eng, us[0], c64[0], raps[0])

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        eng.close()
        return

    total_rays = shard.total_rays(B * RAYS_PER_FRAME, world)
    value = total_rays / (ms_max / 1e3) / 1e6
    plain_value = total_rays / (plain_ms / 1e3) / 1e6
    e2e_value = total_rays / (e2e_ms / 1e3) / 1e6
    # Algorithmic bytes of one launch of the trace kernel (B frames) in the B200 layout: one 72-byte
    # wide node (two child boxes + references) per internal visit, one 80-byte hot record per
    # tetrahedron test, for primary and shadow rays (the visits are the reference traversal's own),
    # plus the 21 bytes of hit record, slot and shadow state written per ray.
    trace_bytes = 72.0 * (work[0] + work[3]) + 80.0 * (work[2] + work[5]) + 21.0 * RAYS_PER_FRAME * B
    trace_s = float(np.median(trace_ms)) / 1e3
    achieved = trace_bytes / trace_s / 1e9
    peak, peak_kind = load_peaks()
    clk = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded accelerated-icosphere scene: no dataset; the reference ships no such scene)",
        "config": workload_config(args, world),
        "rays_per_step": total_rays, "tets": scene.num_prims,
        "footprint": {"scene_device_bytes": int(stats.device_bytes), "fast_nodes": int(stats.fast_nodes),
                      "box_copies": int(stats.box_copies),
                      "layout": "16 sign-octant box copies (SR_LAYOUT_AUTO)" if stats.box_copies == 16 else "compact"},
        "tuning": {k: getattr(tuning, k)
                   for k, _ in tuning._fields_},
        "scene_build_s": round(build_s, 2),
        "plain": {"value": plain_value, "unit": UNIT, "ms_per_step": plain_ms,
                  "speedup_batched_over_plain": value / plain_value},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": (768 + 80) * B,
                "d2h_bytes_per_step": 4 * RAYS_PER_FRAME * B},
        # Kernels per step: camera, trace, shade, 6 bloom down, 5 bloom up, composite.
        "gpu_launches": int(args.steps * 15),
        # The trace kernel is not bound by HBM: its working set (the light cone's share of the
        # tree) is served from L1 and L2, so the byte model below (every node visit and test
        # counted as if fetched) exceeds the HBM roof. What binds it is instruction issue and L1
        # latency (ncu summaries in profiles/); its roof is the same kernel's speed on
        # warp-coherent rays, measured in this run (coherent_roof).
        "roofline": {"bound": "issue", "kernel": "k_trace_lean",
                     **(roof if roof is not None else
                        {"achieved": None, "peak": None, "unit": "Mrays/s", "frac": None,
                         "peak_kind": "not measured (--no-roof, or a scene with stars)"}),
                     "hbm_achieved_gbs": achieved, "hbm_peak_gbs": peak, "hbm_frac": achieved / peak,
                     "hbm_peak_kind": peak_kind,
                     "note": "frac = the trace kernel's time on this batch's counted work at warp-coherent speed "
                             "(fitted on coherent batches in this run) / its measured time: what divergence and "
                             "cache misses cost. hbm_achieved_gbs = algorithmic bytes (72 B per node visit, 80 B "
                             "per tetrahedron test, 21 B written per ray) / trace-kernel time; these bytes are "
                             "mostly served by L1/L2, so hbm_frac > 1 says the kernel is not HBM-bound. DRAM "
                             "traffic and warp-instruction counts come from ncu captures (profiles/), not from "
                             "this run.",
                     "traffic": None,
                     "algorithmic_bytes_per_launch": trace_bytes, "frames_per_launch": B,
                     "trace_ms_per_launch": trace_s * 1e3,
                     "batch_ms": float(np.median(frame_ms)), "shade_ms": float(np.median(shade_ms)),
                     "bloom_ms": float(np.median(bloom_ms)),
                     "per_frame_work": {"node_visits": work[0] / B, "leaf_visits": work[1] / B,
                                        "tet_tests": work[2] / B, "shadow_node_visits": work[3] / B,
                                        "shadow_tet_tests": work[5] / B, "shadow_rays": work[6] / B}},
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
    }
    if compact is not None:
        cs, cms = compact
        line["layout_compact"] = {"value": total_rays / (cms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": cms,
                                  "scene_device_bytes": int(cs.device_bytes), "box_copies": int(cs.box_copies),
                                  "how": "the same batches with SR_LAYOUT_COMPACT: one copy of the child boxes, "
                                         "per-axis min / max in the traversal"}
    if per_ray_ms is not None:
        line["traversal_per_ray"] = {"value": total_rays / (per_ray_ms / 1e3) / 1e6, "unit": UNIT,
                                     "ms_per_step": per_ray_ms,
                                     "how": "the same batches with SrTuning.packet = 0 (each ray walks the tree "
                                            "alone, 128 threads x 11 blocks per SM); the headline walks each "
                                            "tile's rays as a warp packet"}
    if not args.no_extra:
        line["value_fresh"] = {"value": total_rays / (fresh_ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": fresh_ms,
                               "how": "a new seeded set of observers every step, L2 flushed (256 MiB write) before "
                                      "each step, device time of the batches only"}
    line.update(extra)
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(scene.packed(), raps)
        except Exception as exc:  # the baseline is reported, not required for the GPU number
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {exc}"}
    print(json.dumps(line), flush=True)
    eng.close()


def _standalone(args, rank, world, local, fn):
    """One of the extra legs as its own JSON line (config4: observers sharded over ranks)."""
    import torch
    import specrel_b200 as sr
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    eng = sr.Engine(local)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    with ClockSampler(local) as clocks:
        if fn == "config4":
            res = config4_measure(args, rank, world, local, dist, stream, eng, 0)
        else:
            res = config5_measure(args, local, stream, eng, 0) if rank == 0 else None
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    eng.close()
    if rank != 0:
        return
    clk = clocks.summary()
    ms = res.pop("ms_per_step", res["value"])  # config5's value is itself a time
    line = {"metric": res.pop("metric"), "value": res.pop("value"), "unit": res.pop("unit"), "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": res.pop("higher_is_better", True), "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded)", "config": {"workload": res.pop("workload"), "seed": args.seed},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]}}
    line.update(res)
    print(json.dumps(line), flush=True)


def run_tunings(args, local):
    """Trace-kernel time per 8-frame batch of the headline workload under launch settings and node
    layouts (SrTuning fields, sr_set_layout), each timed with the library's CUDA events around the
    kernel outside the captured graph, three rounds interleaved across the settings, medians
    printed as one JSON line. Not a bench line: the comparison behind the default settings."""
    import torch
    import specrel_b200 as sr
    from specrel_b200 import shard
    torch.cuda.set_device(local)
    scene = sr.synth_scene(2, args.seed, n_bodies=args.bodies, threads=os.cpu_count() or 1)
    eng = sr.Engine(local)
    eng.upload(0, scene)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    B = args.batch
    raps = shard.observer_rapidities(args.seed, 0, B, scene.info.cam_rapidity)
    us = [sr.uniforms(sr.camera(rapidity=r), W, H, 0, 1, 0, num_nodes=scene.num_nodes, light_pos=scene.light_pos)
          for r in raps]
    c64 = [sr.cam64((0.0,) * 4, r) for r in raps]
    out = torch.empty(B * RAYS_PER_FRAME, dtype=torch.int32, device=f"cuda:{local}")

    def tune(threads, blocks, stack, top, packet=0):
        t = eng.tuning(0)
        t.block_threads, t.blocks_per_sm, t.stack_smem, t.top_levels, t.packet = threads, blocks, stack, top, packet
        t.tile_w, t.tile_h, t.chunk_tiles, t.refill_lanes, t.leaf_coop, t.leaf_batch, t.home_pct = 4, 8, 1, 32, 0, 1, 0
        eng.set_tuning(0, t)

    def trace_ms(k=5):
        ts = []
        with torch.cuda.stream(stream):
            eng.render_batch(0, us, out.data_ptr(), B * RAYS_PER_FRAME, cams=c64, device_output=True)
            for _ in range(k):
                ts.append(eng.render_batch(0, us, out.data_ptr(), B * RAYS_PER_FRAME, cams=c64, device_output=True,
                                           phases=True).trace_ms)
        return float(np.median(ts))

    L = sr._lib
    cands = [("octant", 128, 11, 0, 0), ("octant", 128, 9, 0, 0), ("octant", 128, 11, 12, 0), ("octant", 128, 9, 12, 0),
             ("octant", 128, 8, 12, 0), ("octant", 128, 9, 10, 0), ("octant", 128, 9, 16, 0), ("octant", 128, 9, 8, 0),
             ("octant", 128, 9, 0, 4), ("octant", 128, 9, 0, 6), ("octant", 128, 9, 0, 8), ("octant", 128, 8, 12, 4),
             ("octant", 128, 8, 12, 6), ("octant", 128, 8, 12, 8), ("compact", 128, 9, 0, 0), ("compact", 128, 9, 10, 0),
             ("octant", 128, 8, 0, 0, 1), ("octant", 256, 4, 0, 0, 1), ("octant", 64, 16, 0, 0, 1),
             ("octant", 128, 6, 0, 0, 1), ("compact", 128, 8, 0, 0, 1)]
    res = {c: [] for c in cands}
    for _ in range(3):
        for layout in ("octant", "compact"):
            eng.set_layout(0, L.SR_LAYOUT_OCTANT if layout == "octant" else L.SR_LAYOUT_COMPACT)
            for c in cands:
                if c[0] == layout:
                    tune(*c[1:])
                    res[c].append(trace_ms())
    eng.set_layout(0, L.SR_LAYOUT_AUTO)
    rows = [{"layout": c[0], "block_threads": c[1], "blocks_per_sm": c[2], "stack_smem": c[3], "top_levels": c[4],
             "packet": c[5] if len(c) > 5 else 0, "trace_ms": float(np.median(v)), "runs": v} for c, v in res.items()]
    print(json.dumps({"what": f"trace-kernel ms per {B}-frame batch, {scene.num_prims} tets, 1280x800", "rows": rows}),
          flush=True)
    eng.close()


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "tunings":
        if rank == 0:
            run_tunings(args, local)
    elif args.workload in ("config4", "config5"):
        _standalone(args, rank, world, local, args.workload)
    else:
        run_engine(args, rank, world, local)


if __name__ == "__main__":
    main()
