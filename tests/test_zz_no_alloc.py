"""sr_render_noalloc: the plain path with all of its scratch in the library's static device array.

Called through the C ABI several times in a row (each call finds the previous call's leftovers in
the shared scratch), every frame must equal sr_render_ex's plain-path frame bit for bit, the
tolerance of the other plain-path parity tests, up to frames at the pixel limit (a 512x512 frame and
the one-row frame of 262,144 pixels, whose bloom pyramid reaches furthest into the scratch). The
device's free memory is the same before and after calls (nothing allocated). Frames above the stated
limit are rejected."""
import ctypes as C

import numpy as np
import pytest

import specrel_b200 as sr
from specrel_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def noalloc_engine():
    eng = sr.Engine(0)
    scene = sr.synth_scene(1, 7, n_bodies=24, steps=16)
    eng.upload(0, scene)
    yield eng, scene
    eng.close()


def _noalloc(eng, u, cam=None):
    import torch
    n = u.size[0] * u.size[1]
    out = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    st = eng.L.sr_render_noalloc(eng.h, 0, C.byref(u), C.byref(cam) if cam is not None else None,
                                 C.c_void_p(out.data_ptr()))
    return st, out.cpu().numpy().view(np.uint32)


def test_calls_in_a_row_match_render_ex(noalloc_engine):
    eng, scene = noalloc_engine
    frames = [
        (sr.camera((0.0, 0.0, 0.0, -4.0), 90.0, rapidity=(0.3, -0.1, 0.2)), 480, 300, None),
        (sr.camera((0.0, 0.0, 0.0, 0.0), 80.0), 256, 160, sr.cam64((0.0, 1.0, -2.0, -6.0), (0.5, 0.2, -0.3))),
    ]
    for cam, w, h, c64 in frames + frames[:1]:
        u = sr.uniforms(cam, w, h, 0, 1, 0, num_nodes=scene.num_nodes, light_pos=scene.light_pos)
        st, got = _noalloc(eng, u, c64)
        assert st == L.SR_OK, eng.L.sr_last_error(eng.h).decode()
        ref = eng.render(0, u, path=sr.SR_PATH_PLAIN, cam=c64).rgb
        assert (got == ref).all()


@pytest.mark.parametrize("w,h", [(512, 512), (L.SR_NOALLOC_MAX_PIXELS, 1), (4096, 64)])
def test_frames_at_the_limit_match_render_ex(noalloc_engine, w, h):
    eng, scene = noalloc_engine
    assert w * h == L.SR_NOALLOC_MAX_PIXELS
    cam = sr.camera((0.0, 0.0, 0.0, -4.0), 90.0, rapidity=(0.3, -0.1, 0.2))
    u = sr.uniforms(cam, w, h, 0, 1, 0, num_nodes=scene.num_nodes, light_pos=scene.light_pos)
    for _ in range(2):
        st, got = _noalloc(eng, u)
        assert st == L.SR_OK, eng.L.sr_last_error(eng.h).decode()
        assert (got == eng.render(0, u, path=sr.SR_PATH_PLAIN).rgb).all()


def test_calls_allocate_no_device_memory(noalloc_engine):
    import torch
    eng, scene = noalloc_engine
    u = sr.uniforms(sr.camera((0.0, 0.0, 0.0, -4.0), 90.0), 512, 512, 0, 1, 0, num_nodes=scene.num_nodes,
                    light_pos=scene.light_pos)
    out = torch.empty(512 * 512, dtype=torch.int32, device="cuda:0")
    call = lambda: eng.L.sr_render_noalloc(eng.h, 0, C.byref(u), None, C.c_void_p(out.data_ptr()))
    assert call() == L.SR_OK  # the library's device code is loaded on the device by now
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        assert call() == L.SR_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_frames_over_the_limit_are_rejected(noalloc_engine):
    eng, scene = noalloc_engine
    u = sr.uniforms(sr.camera(), 640, 480, num_nodes=scene.num_nodes, light_pos=scene.light_pos)
    assert 640 * 480 > L.SR_NOALLOC_MAX_PIXELS
    st, _ = _noalloc(eng, u)
    assert st == L.SR_ERR_INVALID_ARGUMENT
    assert "no-allocation limit" in eng.L.sr_last_error(eng.h).decode()
