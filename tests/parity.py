"""Parity metrics between an engine frame and the CPU oracle (test helper).

The bar: bit-exact hit-tetrahedron ids on non-grazing rays, lambda and tau
within 1e-5 relative, RGB8 within 1/255. Colours may differ only through the last bits of the
transcendentals (CUDA's sinf/cosf/expf/atan2f/acosf against glibc's); a pixel whose oracle
colour changes by more than 1/255 when every transcendental result moves by +-PERTURB ulps is
"near a threshold" and is counted separately rather than compared at 1/255.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from oracle import oracle as O

PERTURB_ULPS = 8
MISS = 0xFFFFFFFF


def channels(rgb: np.ndarray) -> np.ndarray:
    rgb = rgb.astype(np.uint32)
    return np.stack([(rgb >> 16) & 0xFF, (rgb >> 8) & 0xFF, rgb & 0xFF], axis=-1).astype(np.int32)


def rgb_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.abs(channels(a) - channels(b)).max(axis=-1)


@dataclass
class Report:
    n: int
    hit_match: float          # fraction of pixels with the same hit id (miss counts as an id)
    hit_match_nongrazing: float
    grazing_frac: float
    lam_max_rel: float
    tau_max_rel: float
    rgb_max: int
    rgb_max_unmasked: int
    near_threshold_frac: float
    frac_gt1_unmasked: float
    frac_gt4: float           # the reference's own GPU/CPU criterion: < 0.5% of pixels differ by > 4

    def __str__(self):
        return (f"hits {self.hit_match * 100:.4f}% (non-grazing {self.hit_match_nongrazing * 100:.4f}%, grazing "
                f"{self.grazing_frac * 100:.3f}%), lambda rel {self.lam_max_rel:.2e}, tau rel {self.tau_max_rel:.2e}, "
                f"rgb max {self.rgb_max} (unmasked {self.rgb_max_unmasked}), near-threshold "
                f"{self.near_threshold_frac * 100:.3f}%, >1 unmasked {self.frac_gt1_unmasked * 100:.4f}%, "
                f">4 {self.frac_gt4 * 100:.4f}%")


def oracle_frames(scene, cam, cfg, dynamics=None, threads=0):
    base = O.render(scene, cam, cfg, dynamics, threads=threads)
    plus = O.render(scene, cam, cfg, dynamics, threads=threads, perturb=PERTURB_ULPS, aux=False)
    minus = O.render(scene, cam, cfg, dynamics, threads=threads, perturb=-PERTURB_ULPS, aux=False)
    near = (rgb_diff(base.rgb, plus.rgb) > 1) | (rgb_diff(base.rgb, minus.rgb) > 1)
    return base, near


def compare(frame, base, near) -> Report:
    n = base.rgb.size
    gid = frame.hit_id.astype(np.uint32)
    oid = base.orig.astype(np.uint32)
    same = gid == oid
    grazing = (base.slot >= 0) & ((base.min_bary < 1e-4) | (base.denom_rel < 1e-6))
    both = same & (oid != MISS)
    lam_rel = np.abs(frame.lam[both].astype(np.float64) - base.lam[both]) / np.maximum(np.abs(base.lam[both]), 1e-30)
    tau_rel = np.abs(frame.tau[both].astype(np.float64) - base.tau[both]) / np.maximum(np.abs(base.tau[both]), 1.0)
    d = rgb_diff(frame.rgb, base.rgb)
    un = ~near
    return Report(
        n=n,
        hit_match=float(same.mean()),
        hit_match_nongrazing=float(same[~grazing].mean()) if (~grazing).any() else 1.0,
        grazing_frac=float(grazing.mean()),
        lam_max_rel=float(lam_rel.max()) if lam_rel.size else 0.0,
        tau_max_rel=float(tau_rel.max()) if tau_rel.size else 0.0,
        rgb_max=int(d.max()),
        rgb_max_unmasked=int(d[un].max()) if un.any() else 0,
        near_threshold_frac=float(near.mean()),
        frac_gt1_unmasked=float((d[un] > 1).mean()) if un.any() else 0.0,
        frac_gt4=float((d > 4).mean()),
    )


def packed_from_oracle(scene: "O.Scene"):
    """The oracle scene's packed arrays as an engine PackedScene (the caller's data)."""
    import specrel_b200 as sr
    nodes, geoms, attrs, mats, stars, order = scene.pack()
    i = scene.info
    return sr.PackedScene(nodes, geoms, attrs, mats, stars, int(i.n_stars), (0.0, 0.0, 50.0, 0.0), order)
