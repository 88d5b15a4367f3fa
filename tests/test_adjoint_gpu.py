"""The gradient of the image loss with respect to the observer (sr_adjoint), in the star scene's setting:
stars over cube occluders, past light cone, null shadows, loss on the linear pre-bloom HDR image.

Checked against the FP64 CPU reference: the oracle's frozen-outcome loss (oracle/oracle_grad.hpp),
whose central differences at h = 1e-6 give the FP64 gradient and at h = 1e-4 the finite-difference
check; the gradient must match both within 1e-3 (relative, per component against the largest).
Then the rapidity is recovered from zero by gradient descent, coarse to fine over the loss levels."""
import numpy as np
import pytest

import specrel_b200 as sr
from oracle import oracle as O
from parity import packed_from_oracle

pytestmark = pytest.mark.gpu

STAR = (0.8, -0.3, 0.5)
W, H = 160, 100
PARAMS = dict(config=5, seed=2, n_bodies=8, steps=16, n_stars=2000)


@pytest.fixture(scope="module")
def setup(engine):
    import torch
    s32 = O.Scene(O.synth_params(**PARAMS))
    s64 = O.Scene(O.synth_params(**PARAMS), fp64=True)
    engine.upload(11, packed_from_oracle(s32))
    u = sr.uniforms(sr.camera(), W, H, 0, 1, 0, num_nodes=int(s32.info.n_nodes), num_stars=int(s32.info.n_stars))
    tgt = engine.render(11, u, path=sr.SR_PATH_FAST, hdr=True, cam=sr.cam64((0.0, 0.0, 0.0, 0.0), STAR)).hdr
    tdev = torch.tensor(tgt, device="cuda:0").contiguous()
    cfg = O.make_config(W, H, 0, 1, 0)
    t64 = O.render(s64, O.make_camera(rapidity=STAR), cfg, hdr=True, aux=False).hdr
    return dict(u=u, tdev=tdev, s64=s64, cfg=cfg, t64=t64)


def _cam64(th):
    return sr.cam64(tuple(th[3:]), tuple(th[:3]))


def _ocam(th):
    return O.make_camera(pos=tuple(th[3:]), rapidity=tuple(th[:3]))


def _fd(f, th, h):
    return np.array([(f(th + e) - f(th - e)) / (2 * h) for e in np.eye(7) * h])


def _close(g, ref, tol):
    scale = np.abs(ref).max()
    big = np.abs(ref) > 1e-3 * scale
    return bool((np.abs(g - ref) <= tol * scale).all() and (np.abs(g - ref)[big] <= tol * np.abs(ref)[big]).all())


def test_zero_at_the_target(engine, setup):
    r = engine.adjoint(11, setup["u"], sr.cam64((0.0, 0.0, 0.0, 0.0), STAR), setup["tdev"].data_ptr())
    assert r.loss == 0.0 and all(g == 0.0 for g in r.grad)
    assert r.primal_mismatch == 0 and r.star_terms > 1000


@pytest.mark.parametrize("level", [0, 3])
@pytest.mark.parametrize("th0", [(0.75, -0.25, 0.45, 0.0, 0.1, -0.05, 0.08), (0.0,) * 7])
def test_gradient_matches_fp64_reference_and_differences(engine, setup, th0, level):
    th0 = np.array(th0)
    r = engine.adjoint(11, setup["u"], _cam64(th0), setup["tdev"].data_ptr(), level)
    g = np.array(list(r.grad))
    assert r.primal_mismatch == 0  # the recomputed frame equals the forward frame bit for bit
    F = O.Frozen(setup["s64"], _ocam(th0), setup["cfg"])
    loss64 = lambda th: F.loss(_ocam(th), setup["t64"], level)
    assert abs(loss64(th0) - r.loss) <= 1e-4 * r.loss
    ref = _fd(loss64, th0, 1e-6)   # FP64 reference gradient
    fd = _fd(loss64, th0, 1e-4)    # central differences, h = 1e-4
    print("level", level, "gpu", g, "\n fp64", ref, "\n fd", fd)
    assert _close(g, ref, 1e-3)
    assert _close(g, fd, 1e-3)
    # The engine's own f32 loss under the same frozen outcomes agrees too (f32 rounding noise).
    gf = _fd(lambda th: engine.adjoint(11, setup["u"], _cam64(th), setup["tdev"].data_ptr(), level, frozen=True).loss,
             th0, 1e-4)
    assert np.abs(gf - g).max() <= 5e-3 * np.abs(g).max()


def test_frozen_needs_a_gradient_call_first(engine, setup):
    engine.render(11, setup["u"], path=sr.SR_PATH_FAST)  # any frame invalidates the recorded outcomes
    with pytest.raises(sr.SrError):
        engine.adjoint(11, setup["u"], sr.cam64((0.0,) * 4, STAR), setup["tdev"].data_ptr(), frozen=True)


@pytest.mark.parametrize("level", [0, 2])
def test_row_bands_sum_to_the_whole(engine, setup, level):
    """sr_adjoint_rows: the loss, gradient, primal mismatches and star terms of a partition of the
    loss level's rows (as ranks shard them) sum to the whole frame's; the frozen loss of each band
    follows its own gradient call."""
    from specrel_b200 import shard
    th = np.array((0.75, -0.25, 0.45, 0.0, 0.1, -0.05, 0.08))
    u, tp = setup["u"], setup["tdev"].data_ptr()
    whole = engine.adjoint(11, u, _cam64(th), tp, level)
    rows = shard.loss_rows(H, level)
    total = np.zeros(10)
    frozen = 0.0
    for rank in range(3):
        r0, r1 = shard.row_band(rows, rank, 3)
        r = engine.adjoint(11, u, _cam64(th), tp, level, rows=(r0, r1))
        total += [r.loss, *[r.grad[k] for k in range(7)], r.primal_mismatch, r.star_terms]
        frozen += engine.adjoint(11, u, _cam64(th), tp, level, frozen=True, rows=(r0, r1)).loss
    ref = np.array([whole.loss, *[whole.grad[k] for k in range(7)], whole.primal_mismatch, whole.star_terms])
    assert total[8] == ref[8] == 0 and total[9] == ref[9] > 0
    scale = np.abs(ref[1:8]).max()
    assert abs(total[0] - ref[0]) <= 1e-12 * ref[0]
    assert np.abs(total[1:8] - ref[1:8]).max() <= 1e-12 * scale
    assert abs(frozen - ref[0]) <= 1e-12 * ref[0]
    with pytest.raises(sr.SrError):  # a frozen call takes the rows of the gradient call before it
        engine.adjoint(11, u, _cam64(th), tp, level, frozen=True, rows=(0, 1))


def test_gradient_descent_recovers_the_rapidity(engine):
    """The 100k-star scene at 320x200: 100k stars over the cubes; from rapidity 0, normalized gradient descent
    with backtracking on loss levels 6, 5, ..., 0 reaches the target rapidity."""
    import torch
    s = O.Scene(O.synth_params(5, 1, n_bodies=64, steps=64))
    engine.upload(12, packed_from_oracle(s))
    u = sr.uniforms(sr.camera(), 320, 200, 0, 1, 0, num_nodes=int(s.info.n_nodes), num_stars=int(s.info.n_stars))
    ev = (0.0, 0.0, 0.0, 0.0)
    tgt = engine.render(12, u, path=sr.SR_PATH_FAST, hdr=True, cam=sr.cam64(ev, STAR)).hdr
    tdev = torch.tensor(tgt, device="cuda:0").contiguous()

    def lg(phi, level):
        r = engine.adjoint(12, u, sr.cam64(ev, tuple(phi)), tdev.data_ptr(), level)
        return r.loss, np.array(list(r.grad))[:3]

    phi = np.zeros(3)
    for level in range(6, -1, -1):
        step = 0.05
        for _ in range(100):
            L, g = lg(phi, level)
            gn = np.linalg.norm(g)
            if gn == 0:
                break
            moved = False
            while step > 1e-8:
                cand = phi - step * g / gn
                if lg(cand, level)[0] < L:
                    phi, step, moved = cand, step * 1.5, True
                    break
                step *= 0.5
            if not moved:
                break
    print("recovered", phi)
    assert np.abs(phi - np.array(STAR)).max() < 1e-4


def test_group_gradient_through_the_c_abi(engine, setup):
    """sr_adjoint_group, the path a non-Python host takes over several GPUs, run as three ranks in
    turn on this GPU with a sum that records each rank's part: the parts sum to sr_adjoint's whole
    frame. Then as a group of one over a real NCCL communicator through sr_nccl_sum_f64."""
    import ctypes as C

    import torch
    from specrel_b200 import _lib as L
    th = np.array((0.75, -0.25, 0.45, 0.0, 0.1, -0.05, 0.08))
    u, cam, tp = setup["u"], _cam64(th), setup["tdev"].data_ptr()
    whole = engine.adjoint(11, u, cam, tp, 2)
    parts = []

    @L.SUM_F64_FN
    def record(values, count, user):
        parts.append(np.ctypeslib.as_array(values, shape=(count,)).copy())
        return 0

    for rank in range(3):
        r = L.AdjointResult()
        assert engine.L.sr_adjoint_group(engine.h, 11, C.byref(u), C.byref(cam), tp, 2, 0, rank, 3, record, None,
                                         C.byref(r)) == L.SR_OK
    total = np.sum(parts, axis=0)
    ref = np.array([whole.loss, *[whole.grad[k] for k in range(7)], whole.primal_mismatch, whole.star_terms])
    assert len(parts) == 3
    assert abs(total[0] - ref[0]) <= 1e-12 * ref[0]
    assert np.abs(total[1:8] - ref[1:8]).max() <= 1e-12 * np.abs(ref[1:8]).max()
    assert total[8] == ref[8] and total[9] == ref[9]

    # A group of one over NCCL (the communicator made here through NCCL's own C API).
    nccl = C.CDLL("libnccl.so.2")

    class UniqueId(C.Structure):
        _fields_ = [("internal", C.c_char * 128)]

    uid = UniqueId()
    assert nccl.ncclGetUniqueId(C.byref(uid)) == 0
    comm = C.c_void_p()
    assert nccl.ncclCommInitRank(C.byref(comm), 1, uid, 0) == 0
    try:
        buf = torch.zeros(10, dtype=torch.float64, device="cuda:0")
        s = L.NcclSum(comm, None, buf.data_ptr())
        nccl_sum = L.SUM_F64_FN(("sr_nccl_sum_f64", engine.L))
        r = L.AdjointResult()
        assert engine.L.sr_adjoint_group(engine.h, 11, C.byref(u), C.byref(cam), tp, 2, 0, 0, 1, nccl_sum, C.byref(s),
                                         C.byref(r)) == L.SR_OK
        assert r.loss == whole.loss and list(r.grad) == list(whole.grad)
    finally:
        nccl.ncclCommDestroy(comm)
