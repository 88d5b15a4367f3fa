"""The oracle against the committed golden fixtures (tests/golden, made by make_golden.py): the
oracle build on this machine must reproduce every fixture bit for bit (hit ids, lambda, tau, RGB),
so the fixtures pin the checker the GPU parity tests rely on."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import CASES  # noqa: E402
from oracle import oracle as O  # noqa: E402


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_fixture(name):
    sp, fp64, cam, (w, h, mode, shadow, slice_) = CASES[name]
    g = load(name)
    scene = O.Scene(O.synth_params(**sp), fp64=fp64)
    r = O.render(scene, O.make_camera(**cam), O.make_config(w, h, mode, shadow, slice_))
    dt = np.float64 if fp64 else np.float32
    assert (r.orig.astype(np.uint32) == g["orig"]).all()
    assert (r.lam.astype(dt) == g["lam"]).all()
    assert (r.tau.astype(dt) == g["tau"]).all()
    assert (r.rgb.astype(np.uint32) == g["rgb"]).all()
    assert (g["orig"] != 0xFFFFFFFF).sum() > 200
