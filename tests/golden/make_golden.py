"""Generates the golden fixtures of tests/golden from the oracle (the C++ restatement of the
reference's renderer, pinned by the reference's own known-answer tests in oracle/oracle_kat.cpp).

Each case is a small seeded frame of one of the workloads, rendered by the oracle; the fixture
keeps per pixel the hit's original simplex id, lambda, tau, the packed RGB and the near-threshold
mask (pixels whose colour moves by more than 1/255 when every transcendental moves by +-8 ulps).

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402

# name -> (synth_params args, fp64, camera kwargs, (width, height, mode, shadow_mode, slice_mode))
CASES = {
    "config1_cubes_160x100": (dict(config=1, seed=2), False,
                              dict(pos=(0.0, 0.0, 0.0, -4.0), rapidity=(0.3, 0.1, -0.2), fov_deg=120.0),
                              (160, 100, 0, 1, 0)),
    "config2_spheres24_160x100": (dict(config=2, seed=4, n_bodies=24, steps=32), False,
                                  dict(pos=(0.0, 0.0, 0.0, 0.0), rapidity=(0.4, -0.2, 0.1)), (160, 100, 0, 1, 0)),
    "config3_translated_fp64_160x100": (dict(config=3, seed=1), True,
                                        dict(pos=(1e6, 6e4, 0.0, 8e4)), (160, 100, 0, 0, 0)),
    "config5_stars2000_160x100": (dict(config=5, seed=3, n_stars=2000), False,
                                  dict(pos=(0.0, 0.0, 0.0, 0.0), rapidity=(0.8, -0.3, 0.5)), (160, 100, 0, 0, 0)),
}


def render_case(name):
    from parity import oracle_frames
    sp, fp64, cam, (w, h, mode, shadow, slice_) = CASES[name]
    scene = O.Scene(O.synth_params(**sp), fp64=fp64)
    cfg = O.make_config(w, h, mode, shadow, slice_)
    base, near = oracle_frames(scene, O.make_camera(**cam), cfg)
    dt = np.float64 if fp64 else np.float32
    return dict(orig=base.orig.astype(np.uint32), lam=base.lam.astype(dt), tau=base.tau.astype(dt),
                rgb=base.rgb.astype(np.uint32), near=near.astype(bool))


def main():
    for name in CASES:
        arrays = render_case(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        hits = int((arrays["orig"] != 0xFFFFFFFF).sum())
        print(f"{name}: {hits} hits of {arrays['orig'].size}, near-threshold {int(arrays['near'].sum())}")


if __name__ == "__main__":
    main()
