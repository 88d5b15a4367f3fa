"""The scene build on the device. sr_build_scene: Bvh4D::build and the leaf-order packing run on the
GPU from the simplices in build order; sr_build_scene_tubes: the worldtubes' simplices extruded on
the GPU too. The node array, the leaf order and the records must equal the host build's byte for
byte (the host builder is itself bit-exact with the oracle's restatement of the reference's build),
and frames rendered from the device-built scene must equal frames from the uploaded one."""
import os
import time

import numpy as np
import pytest

import specrel_b200 as sr

pytestmark = pytest.mark.gpu

CASES = [
    dict(config=1, seed=1),
    dict(config=1, seed=2),
    dict(config=2, seed=4, n_bodies=24, steps=24),
    dict(config=5, seed=1, n_stars=2000),
]


def _build_and_compare(engine, idx, scene):
    boxes, geoms, attrs, p = scene.build_inputs()
    t0 = time.perf_counter()
    engine.build(idx, boxes, geoms, attrs, p.materials, p.stars, p.num_stars, p.light_pos, p.anchor)
    t_gpu = time.perf_counter() - t0
    nodes, order = engine.tree(idx)
    assert len(nodes) == len(p.nodes)
    assert nodes.tobytes() == p.nodes.tobytes()
    assert (order == p.leaf_to_orig).all()
    return t_gpu


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_device_build_equals_host_build(engine, case):
    scene = sr.synth_scene(**case)
    t_gpu = _build_and_compare(engine, 21, scene)
    print(case, "prims", scene.num_prims, "nodes", scene.num_nodes, f"host build {scene.info.build_seconds:.3f} s,"
          f" device build (with uploads) {t_gpu:.3f} s")
    # Frames from the device-built scene equal frames from the uploaded scene.
    engine.upload(22, scene)
    u = sr.uniforms(sr.camera(rapidity=tuple(scene.info.cam_rapidity)), 320, 200, 0, 1, 0,
                    num_nodes=scene.num_nodes, num_stars=scene.num_stars)
    for path in (sr.SR_PATH_FAST, sr.SR_PATH_PLAIN):
        a = engine.render(21, u, path=path, aux=True)
        b = engine.render(22, u, path=path, aux=True)
        assert (a.rgb == b.rgb).all() and (a.hit_id == b.hit_id).all() and (a.lam == b.lam).all()


def _tubes_and_compare(engine, idx, scene):
    p = scene.packed()
    t0 = time.perf_counter()
    engine.build_tubes(idx, scene)
    t_gpu = time.perf_counter() - t0
    nodes, order = engine.tree(idx)
    g, a = engine.records(idx)
    assert nodes.tobytes() == p.nodes.tobytes()
    assert (order == p.leaf_to_orig).all()
    assert g.tobytes() == p.geoms.tobytes() and a.tobytes() == p.attrs.tobytes()
    return t_gpu


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_device_extrusion_and_build_equal_host_build(engine, case):
    scene = sr.synth_scene(**case)
    t_gpu = _tubes_and_compare(engine, 23, scene)
    print(case, f"tubes built on the device in {t_gpu:.3f} s")
    engine.upload(22, scene)
    u = sr.uniforms(sr.camera(rapidity=tuple(scene.info.cam_rapidity)), 320, 200, 0, 1, 0,
                    num_nodes=scene.num_nodes, num_stars=scene.num_stars)
    a = engine.render(23, u, path=sr.SR_PATH_FAST, aux=True)
    b = engine.render(22, u, path=sr.SR_PATH_FAST, aux=True)
    assert (a.rgb == b.rgb).all() and (a.hit_id == b.hit_id).all()


def test_device_build_full_size(engine):
    """The icosphere scene at full size: 7.9M simplices, from build-order simplices and from worldtubes."""
    scene = sr.synth_scene(2, 1, threads=os.cpu_count())
    t_gpu = _build_and_compare(engine, 21, scene)
    t_tubes = _tubes_and_compare(engine, 23, scene)
    print("7.9M tets: host build", f"{scene.info.build_seconds:.2f} s (synthesis, extrusion and tree, host threads),",
          f"device build {t_gpu:.3f} s from simplices (uploads, tree, leaf order, node layout),",
          f"{t_tubes:.3f} s from worldtubes (extrusion included)")


def test_device_extrusion_flags_tubes_past_their_rindler_horizon(engine):
    """The sampled accelerations of the icosphere scene's bodies carry the reference's f32 finite-difference
    noise, which crosses 1 + a_local . p > 0 for vertices of some larger bodies (the host builder
    records it as rindler_ok = 0): the device build extrudes them all the same and flags it."""
    for case in (dict(config=2, seed=4, n_bodies=24, steps=24), dict(config=1, seed=1)):
        scene = sr.synth_scene(**case)
        engine.build_tubes(27, scene)
        assert engine.stats(27).rindler_crossed == (0 if scene.info.rindler_ok else 1), case


def test_device_build_rejects_empty(engine):
    with pytest.raises(sr.SrError):
        engine.build(21, np.zeros((0, 8), np.float32), np.zeros(0, sr.GEOM_DTYPE), np.zeros(0, sr.ATTR_DTYPE),
                     sr.synth_scene(1, 1).packed().materials)


def test_dynamic_scale_update_and_rebuild(engine):
    """The per-frame scene cost of the reference's dynamic mode, at its quoted size (about 12.5k
    simplices): a dirty-range update of every array (sr_update_scene) and a full rebuild from the
    worldtubes on the device (sr_build_scene_tubes), each timed on the host around the call; both
    render as a fresh upload does."""
    scene = sr.synth_scene(1, 3, n_bodies=16, steps=22)
    p = scene.packed()
    engine.upload(24, scene)
    u = sr.uniforms(sr.camera(rapidity=tuple(scene.info.cam_rapidity)), 320, 200, 0, 1, 0, num_nodes=scene.num_nodes)
    ref = engine.render(24, u, path=sr.SR_PATH_FAST).rgb
    ts_up, ts_build = [], []
    for _ in range(10):
        t0 = time.perf_counter()
        engine.update(24, scene, node_ranges=[(0, len(p.nodes))], prim_ranges=[(0, len(p.geoms))])
        ts_up.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        engine.build_tubes(25, scene)
        ts_build.append(time.perf_counter() - t0)
    assert (engine.render(24, u, path=sr.SR_PATH_FAST).rgb == ref).all()
    assert (engine.render(25, u, path=sr.SR_PATH_FAST).rgb == ref).all()
    print(f"{scene.num_prims} simplices: dirty-range update {np.median(ts_up) * 1e3:.2f} ms, "
          f"rebuild from worldtubes on the device {np.median(ts_build) * 1e3:.2f} ms (medians of 10)")


def test_device_build_reports_the_median_split(engine):
    """A node whose SAH split leaves one side empty is split at the centroid median by the reference
    (Rust's select_nth_unstable_by); the device build does not restate that selection and returns
    SR_ERR_UNSUPPORTED, so such a scene is built on the host (sr_bvh_build_host flags it)."""
    from test_median_split import degenerate_boxes, host_build
    boxes = degenerate_boxes()
    n = len(boxes)
    mats = sr.synth_scene(1, 1, n_bodies=2, steps=2).packed().materials
    with pytest.raises(sr.SrError) as e:
        engine.build(22, boxes, np.zeros(n, sr.GEOM_DTYPE), np.zeros(n, sr.ATTR_DTYPE), mats)
    assert e.value.status == sr._lib.SR_ERR_UNSUPPORTED
    assert host_build(boxes)[2] == 1
