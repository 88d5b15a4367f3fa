"""The BVH build's median split (bvh4d.rs:418-424): when the SAH partition leaves one side empty,
the reference reorders the node's items with Rust's slice::select_nth_unstable_by, and the tree below
depends on the order that leaves. The oracle and the library's host builder both restate that
selection (Rust 1.81+'s partition_at_index); Rust itself cannot run here, so the restatement is held
to what the selection guarantees and to its deterministic pieces, and the two builders to each
other on a scene that takes the fallback."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("n", [2, 5, 16, 17, 40, 63, 64, 65, 300, 1500, 5000])
def test_selection_property_and_permutation(n):
    rng = np.random.default_rng(n)
    for trial in range(6):
        keys = rng.integers(0, max(2, n // (1 + trial)), n).astype(np.float32)  # many ties on later trials
        for k in sorted({0, n - 1, n // 2, rng.integers(0, n)}):
            v, idx = O.select_nth(keys, k)
            assert sorted(idx) == list(range(n))
            assert (keys[idx] == v).all()
            assert (v[:k] <= v[k]).all() and (v[k + 1:] >= v[k]).all()


@pytest.mark.parametrize("n", [3, 7, 12, 16])
def test_small_slices_are_insertion_sorted(n):
    """Up to 16 elements the selection is an insertion sort: a stable sort of the slice."""
    rng = np.random.default_rng(7 + n)
    keys = rng.integers(0, 4, n).astype(np.float32)
    for k in range(1, n - 1):
        v, idx = O.select_nth(keys, k)
        ref = np.argsort(keys, kind="stable")
        assert (idx == ref).all()


def test_ends_swap_the_first_extreme():
    """k = 0 swaps the first minimum to the front, k = n - 1 the first maximum to the back
    (min_index / max_index keep the earlier of equal elements)."""
    keys = np.array([3, 1, 4, 1, 5, 9, 2, 6, 5, 3, 9, 1] * 3, np.float32)
    v, idx = O.select_nth(keys, 0)
    assert idx[0] == 1 and idx[1] == 0 and (idx[2:] == np.arange(2, len(keys))).all()
    v, idx = O.select_nth(keys, len(keys) - 1)
    assert idx[-1] == 5 and idx[5] == len(keys) - 1


def degenerate_boxes(n=300, seed=3):
    """Boxes whose centroids take two values one f32 step apart near t = 1000: the spread (6.1e-5)
    is below the SAH's 1e-4, so the split falls to the centre of the centroid box, which rounds onto
    the lower value; no centroid is below it, so the reference selects by median."""
    lo = np.float32(1000.0)
    hi = np.nextafter(lo, np.float32(2000.0))
    rng = np.random.default_rng(seed)
    c = np.where(rng.random(n) < 0.5, lo, hi).astype(np.float32)
    c[: n // 2], c[n // 2:] = lo, hi  # exactly half of each ...
    rng.shuffle(c)                    # ... in a mixed order
    b = np.zeros((n, 8), np.float32)
    b[:, 0], b[:, 4] = c - np.float32(1), c + np.float32(1)  # centre (c - 1 + c + 1) / 2 == c
    w = rng.random(n).astype(np.float32)                       # distinct boxes, equal centres
    for a in (1, 2, 3):
        b[:, a], b[:, 4 + a] = np.float32(0.5) - w, np.float32(0.5) + w
    return b


def host_build(boxes):
    from specrel_b200 import _lib as L
    n = len(boxes)
    nodes = np.zeros(2 * n - 1, L.NODE_DTYPE)
    order = np.zeros(n, np.uint32)
    nn, med = C.c_uint32(), C.c_uint32()
    b = np.ascontiguousarray(boxes, np.float32)
    assert L.lib().sr_bvh_build_host(b.ctypes.data, n, 4, nodes.ctypes.data, len(nodes), order.ctypes.data,
                                     C.byref(nn), C.byref(med)) == L.SR_OK
    return nodes[:nn.value], order, med.value


def test_degenerate_centroids_take_the_median_split():
    boxes = degenerate_boxes()
    onodes, oorder, omed = O.bvh_from_boxes(boxes)
    hnodes, horder, hmed = host_build(boxes)
    assert omed == 1 and hmed == 1
    assert (onodes.tobytes() == hnodes.tobytes()) and (oorder == horder).all()
    # Root and two leaves: the lower centroids on the left, in the selection's order.
    assert len(onodes) == 3 and onodes["count"][0] == 0 and onodes["count"][1] == 150 and onodes["count"][2] == 150
    c = (boxes[:, 0] + boxes[:, 4]) * np.float32(0.5)
    assert (c[oorder[:150]] < c[oorder[150:]].min()).all()
    assert sorted(oorder) == list(range(len(boxes)))


def test_the_workloads_never_take_the_median_split():
    import specrel_b200 as sr
    for cfg, kw in ((1, {}), (2, dict(n_bodies=12, steps=24)), (5, dict(n_bodies=8, steps=16))):
        assert sr.synth_scene(cfg, 1, **kw).info.median_splits == 0
        assert O.Scene(O.synth_params(cfg, 1, **kw)).info.median_splits == 0
