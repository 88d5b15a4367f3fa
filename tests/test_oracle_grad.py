"""The oracle's frozen-outcome loss (the FP64 reference of the engine's gradient): at the observer it
was frozen at, it reproduces the oracle's own render exactly; it is smooth around it, so central
differences at h = 1e-4 and h = 1e-6 agree."""
import numpy as np

from oracle import oracle as O


def test_frozen_frame_reproduces_the_render_and_is_smooth():
    s = O.Scene(O.synth_params(5, 2, n_bodies=8, steps=16, n_stars=2000), fp64=True)
    cfg = O.make_config(160, 100, 0, 1, 0)
    tgt = O.render(s, O.make_camera(rapidity=(0.8, -0.3, 0.5)), cfg, hdr=True, aux=False).hdr
    th0 = np.array([0.75, -0.25, 0.45, 0.0, 0.1, -0.05, 0.08])
    cam = lambda th: O.make_camera(pos=tuple(th[3:]), rapidity=tuple(th[:3]))
    F = O.Frozen(s, cam(th0), cfg)
    L0, img = F.loss(cam(th0), tgt, 0, hdr=True)
    ref = O.render(s, cam(th0), cfg, hdr=True, aux=False).hdr
    assert (img == ref).all()
    assert L0 == ((ref - tgt) ** 2).sum() or abs(L0 - ((ref - tgt) ** 2).sum()) <= 1e-12 * L0
    g4 = np.array([(F.loss(cam(th0 + e), tgt) - F.loss(cam(th0 - e), tgt)) / 2e-4 for e in np.eye(7) * 1e-4])
    g6 = np.array([(F.loss(cam(th0 + e), tgt) - F.loss(cam(th0 - e), tgt)) / 2e-6 for e in np.eye(7) * 1e-6])
    assert np.abs(g4 - g6).max() <= 1e-3 * np.abs(g6).max()
    # A coarser loss level is smaller and still differentiable.
    assert F.loss(cam(th0), tgt, 3) < L0


def test_binned_freeze_records_the_same_outcomes():
    """Large star sets find each pixel's candidate stars by projection instead of testing every star;
    the frozen image (every star that passed the footprint cut, in the same order) is the same."""
    s = O.Scene(O.synth_params(5, 3, n_bodies=4, steps=8, n_stars=20000), fp64=True)
    cfg = O.make_config(200, 125, 0, 1, 0)
    th0 = np.array([0.3, -0.2, 0.1, 0.0, 0.05, 0.0, -0.02])
    cam = O.make_camera(pos=tuple(th0[3:]), rapidity=tuple(th0[:3]))
    tgt = np.zeros((200 * 125, 3))
    L0, a = O.Frozen(s, cam, cfg, binning=0).loss(cam, tgt, hdr=True)
    L1, b = O.Frozen(s, cam, cfg, binning=1).loss(cam, tgt, hdr=True)
    ref = O.render(s, cam, cfg, hdr=True, aux=False).hdr
    assert (a == ref).all() and (b == ref).all() and L0 == L1
