"""The gradient at the star workload's stated size: 100k inertial point stars on a sphere of radius
1e3 over the 64 cube occluders, 1280x800, past light cone, null shadows; the target rendered at
rapidity (0.8, -0.3, 0.5), the gradient taken where bench.py times it (rapidity 0, event 0) and
near the target.

Checked against the FP64 CPU reference: the oracle's frozen-outcome loss in double (scene built in
double, the discrete outcomes recorded at the same observer), whose central differences at
h = 1e-6 give the FP64 gradient, and whose central differences at h = 1e-4 give the
finite-difference check. At this resolution a star's footprint is one pixel pitch (2.5e-3 rad)
wide, so h = 1e-4 is 4% of it and the second-order difference (f(x + h) - f(x - h)) / 2h carries a
truncation error of about 1% (measured 1.1e-2); the check uses the fourth-order central difference
at the same h, (-f(x + 2h) + 8 f(x + h) - 8 f(x - h) + f(x - 2h)) / 12h, and prints both. Both sides
use the engine's target image. The gradient must match the FP64 gradient and the differences within
1e-3 relative (per component against the largest, and per component where it is above 1e-3 of the
largest)."""
import os

import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import packed_from_oracle

pytestmark = pytest.mark.gpu

STAR = (0.8, -0.3, 0.5)
W, H = 1280, 800
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def full(engine):
    import torch
    s32 = O.Scene(O.synth_params(5, 1))
    assert int(s32.info.n_stars) == 100000
    s64 = O.Scene(O.synth_params(5, 1), fp64=True)
    engine.upload(31, packed_from_oracle(s32))
    u = sr.uniforms(sr.camera(), W, H, 0, 1, 0, num_nodes=int(s32.info.n_nodes), num_stars=int(s32.info.n_stars))
    tgt = engine.render(31, u, path=sr.SR_PATH_FAST, hdr=True, cam=sr.cam64((0.0, 0.0, 0.0, 0.0), STAR)).hdr
    tdev = torch.tensor(tgt, device="cuda:0").contiguous()
    return dict(u=u, tdev=tdev, s64=s64, cfg=O.make_config(W, H, 0, 1, 0), t64=tgt[:, :3].astype(np.float64))


def _cam64(th):
    return sr.cam64(tuple(th[3:]), tuple(th[:3]))


def _ocam(th):
    return O.make_camera(pos=tuple(th[3:]), rapidity=tuple(th[:3]))


def _fd(f, th, h):
    return np.array([(f(th + e) - f(th - e)) / (2 * h) for e in np.eye(7) * h])


def _fd4(f, th, h):
    return np.array([(-f(th + 2 * e) + 8 * f(th + e) - 8 * f(th - e) + f(th - 2 * e)) / (12 * h) for e in np.eye(7) * h])


def _close(g, ref, tol):
    scale = np.abs(ref).max()
    big = np.abs(ref) > 1e-3 * scale
    return bool((np.abs(g - ref) <= tol * scale).all() and (np.abs(g - ref)[big] <= tol * np.abs(ref)[big]).all())


@pytest.mark.parametrize("th0", [(0.0,) * 7, (0.75, -0.25, 0.45, 0.0, 0.1, -0.05, 0.08)])
def test_full_size_gradient_matches_fp64_reference_and_differences(engine, full, th0):
    th0 = np.array(th0)
    r = engine.adjoint(31, full["u"], _cam64(th0), full["tdev"].data_ptr(), 0)
    g = np.array(list(r.grad))
    assert r.primal_mismatch == 0  # the recomputed frame equals the forward frame bit for bit
    assert r.star_terms > 100000
    F = O.Frozen(full["s64"], _ocam(th0), full["cfg"], threads=THREADS)
    loss64 = lambda th: F.loss(_ocam(th), full["t64"], 0, threads=THREADS)
    L64 = loss64(th0)
    ref = _fd(loss64, th0, 1e-6)   # FP64 reference gradient
    fd2 = _fd(loss64, th0, 1e-4)   # second-order central differences, h = 1e-4 (reported)
    fd = _fd4(loss64, th0, 1e-4)   # fourth-order central differences, h = 1e-4 (checked)
    rel = lambda a, b: np.abs(a - b).max() / np.abs(b).max()
    print(f"1280x800, 100k stars, theta0 {tuple(th0)}: loss gpu {r.loss:.9e} fp64 {L64:.9e}, star terms "
          f"{int(r.star_terms)}\n gpu  {g}\n fp64 {ref}\n fd4  {fd}\n fd2  {fd2}\n max rel diff: fp64 {rel(g, ref):.2e}, "
          f"fd4 {rel(g, fd):.2e}, fd2 {rel(g, fd2):.2e}")
    assert abs(L64 - r.loss) <= 1e-4 * r.loss
    assert _close(g, ref, 1e-3)
    assert _close(g, fd, 1e-3)
