"""The C ABI: the library loads without a GPU, exports every function the headers declare, its
structs have the reference's layouts, and the host-side scene checks reject bad input."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in ("specrel.h", "specrel_scene.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(sr_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    import specrel_b200._lib as L
    lib = C.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert names == set(L.SIGNATURES), sorted(names ^ set(L.SIGNATURES))


def test_struct_layouts_match_the_reference():
    import specrel_b200._lib as L
    assert L.NODE_DTYPE.itemsize == 48       # GpuNode, gpu.rs:44-51
    assert L.GEOM_DTYPE.itemsize == 80       # GpuGeom, gpu.rs:68-74
    assert L.ATTR_DTYPE.itemsize == 192      # GpuAttr, gpu.rs:79-92
    assert L.MAT_DTYPE.itemsize == 48        # GpuMaterial, gpu.rs:96-100
    assert C.sizeof(L.GpuUniforms) == 768    # GpuUniforms, gpu.rs:122-144
    U = L.GpuUniforms
    offs = {"light_pos": 80, "num_nodes": 124, "frontier_origin": 128, "frontier_view_offset": 144,
            "num_flashes": 148, "frontier_tau": 152, "num_haze": 160, "num_stars": 164, "haze_origin": 176,
            "flash_at": 256, "flash_col_width": 512}
    for k, v in offs.items():
        assert getattr(U, k).offset == v, k
    assert L.ATTR_DTYPE.fields["misc"][1] == 160 and L.ATTR_DTYPE.fields["decided_at"][1] == 176
    assert C.sizeof(L.Tuning) == 48 and L.Tuning.leaf_coop.offset == 24 and L.Tuning.home_pct.offset == 32
    assert C.sizeof(L.Timings) == 96
    assert L.TRI_DTYPE.itemsize == 48 and L.SAMPLE_DTYPE.itemsize == 112 and C.sizeof(L.Tube) == 48
    assert C.sizeof(L.ArenaPart) == 16 and C.sizeof(L.ArenaStats) == 48 and L.Tube.decided_at.offset == 40


def test_create_without_device_fails_cleanly():
    import specrel_b200 as sr
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(sr.SrError) as e:
        sr.Engine(0)
    assert e.value.status == sr._lib.SR_ERR_NO_DEVICE


def _tiny_scene():
    import specrel_b200 as sr
    s = sr.synth_scene(1, 3, n_bodies=2, steps=2)
    return s.packed()


def test_validate_accepts_built_scene():
    import specrel_b200 as sr
    p = _tiny_scene()
    st, depth, msg = sr.validate(p)
    assert st == 0, msg
    assert depth >= 2


@pytest.mark.parametrize("breakage", ["child_out_of_range", "cycle", "leaf_range", "material", "order", "star"])
def test_validate_rejects_corrupt_scene(breakage):
    import specrel_b200 as sr
    p = _tiny_scene()
    nodes = p.nodes.copy()
    internal = np.nonzero(nodes["count"] == 0)[0]
    leaves = np.nonzero(nodes["count"] > 0)[0]
    if breakage == "child_out_of_range":
        nodes["left"][internal[0]] = len(nodes) + 5
    elif breakage == "cycle":
        nodes["right_or_first"][internal[-1]] = 0
    elif breakage == "leaf_range":
        nodes["right_or_first"][leaves[0]] = len(p.geoms)
    elif breakage == "material":
        attrs = p.attrs.copy()
        attrs["misc"][0, 2] = np.uint32(99).view(np.float32)
        p.attrs = attrs
    elif breakage == "order":
        p.leaf_to_orig = p.leaf_to_orig.copy()
        p.leaf_to_orig[3] = len(p.geoms) + 1
    elif breakage == "star":
        st = np.zeros(4 + 12, np.float32)
        st[2] = np.uint32(0).view(np.float32)
        st[3] = np.uint32(2).view(np.float32)  # two segments, only one present
        p.stars = st
        p.num_stars = 1
    p.nodes = nodes
    status, _, msg = sr.validate(p)
    assert status == sr._lib.SR_ERR_BAD_SCENE, breakage
    assert msg


C_PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "specrel.h"
#include "specrel_scene.h"

/* A non-Python host: one leaf holding one tetrahedron, validated on the host, then a context. */
int main(void) {
    SrGpuNode node;
    memset(&node, 0, sizeof node);
    for (int k = 0; k < 4; ++k) { node.min[k] = -1.0f; node.max[k] = 1.0f; }
    node.right_or_first = 0;
    node.count = 1;
    SrGpuGeom geom;
    SrGpuAttr attr;
    memset(&geom, 0, sizeof geom);
    memset(&attr, 0, sizeof attr);
    SrGpuMaterial mat;
    memset(&mat, 0, sizeof mat);
    SrSceneDesc d;
    memset(&d, 0, sizeof d);
    d.nodes = &node;
    d.num_nodes = 1;
    d.num_prims = 1;
    d.geoms = &geom;
    d.attrs = &attr;
    d.materials = &mat;
    d.num_materials = 1;
    uint32_t depth = 0;
    char err[256] = "";
    sr_status v = sr_scene_validate(&d, &depth, err, sizeof err);
    node.count = 2; /* a leaf past the records */
    sr_status bad = sr_scene_validate(&d, NULL, err, sizeof err);
    sr_ctx* ctx = NULL;
    char cerr[256] = "";
    sr_status c = sr_create(0, &ctx, cerr, sizeof cerr);
    if (c == SR_OK) sr_destroy(ctx);
    uint32_t r0 = 0, r1 = 0;
    sr_status b = sr_adjoint_band(800, 3, 1, 4, &r0, &r1);
    printf("%d %u %d %d %d %u %u\n", (int)v, depth, (int)bad, (int)c, (int)b, r0, r1);
    return 0;
}
"""


def test_c_host_compiles_links_and_calls_the_library(tmp_path):
    """A C program built with gcc against include/specrel.h and include/specrel_scene.h (C99), linked
    with libspecrel_cuda.so, calls the library as a Rust or C host would: host-side validation, a
    context (SR_ERR_NO_DEVICE without a GPU) and the gradient's row bands."""
    import subprocess
    import specrel_b200._lib as L
    src = tmp_path / "host.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "host"
    libdir = os.path.dirname(L.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lspecrel_cuda", f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    v, depth, bad, c, b, r0, r1 = map(int, out)
    assert v == L.SR_OK and depth == 1
    assert bad == L.SR_ERR_BAD_SCENE
    import torch
    assert c == (L.SR_OK if torch.cuda.is_available() else L.SR_ERR_NO_DEVICE)
    assert b == L.SR_OK and (r0, r1) == (25, 50)  # 800 rows halved 3 times: 100, rank 1 of 4
