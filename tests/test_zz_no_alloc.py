"""The allocation-free join entry point (vs_join_brute_noalloc).

It serves callers that cannot allocate device memory: hosts that own every
byte of device memory in a fixed arena, processes on a hard memory budget,
or loops that cannot pay for an allocation's synchronisation.  Its only
scratch is a fixed device array inside the library, shared by every call.

This file is collected last on purpose, so that a run that stops at the first
failure has already run every other test.  The check: two calls in a row
through the C-ABI return exactly the pair set of the regular entry point
(vs_join, brute method), and inputs above the fixed limit are rejected.
"""
import numpy as np
import pytest

from _helpers import PRED_CODES, gpu_join, upload_points, upload_polys

pytestmark = pytest.mark.gpu


def _sorted_pairs(l, r):
    o = np.lexsort((r, l))
    return l[o], r[o]


@pytest.mark.parametrize("predicate", ["within", "intersects", None])
def test_noalloc_matches_vs_join_twice(vsabi, ctx, predicate):
    import torch
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=21, n_points=40_000, n_polys=800)
    el, er, _ = gpu_join(vsabi, ctx, w.px, w.py, w.polys, predicate, method=2)  # existing entry point
    pts, keep_pts = upload_points(vsabi, w.px, w.py)
    polys, keep_polys = upload_polys(vsabi, w.polys)
    cap = len(el) + 16
    for _ in range(2):  # the shared scratch keeps the last call's contents: the second call must not see them
        left = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        right = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        n = vsabi.join_brute_noalloc(pts, polys, PRED_CODES[predicate], left, right)
        gl, gr = _sorted_pairs(left[:n].cpu().numpy(), right[:n].cpu().numpy())
        assert n == len(el)
        np.testing.assert_array_equal(gl, el)
        np.testing.assert_array_equal(gr, er)


def test_noalloc_rejects_inputs_over_the_limit(vsabi):
    from vibespatial_b200 import _abi

    # 65,537 polygon rows: refused before any device work
    P = _abi.Polygons(0, 0, 1, 1, 1, None, 0, 0, 0, 65_537)
    pts = _abi.Points(1, 1, None, 10)
    with pytest.raises(ValueError, match="at most 65536 polygons"):
        _abi.join_brute_noalloc(pts, P, PRED_CODES["within"], None, None)


def test_noalloc_capacity_error(vsabi):
    import torch
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=22, n_points=20_000, n_polys=300)
    pts, keep_pts = upload_points(vsabi, w.px, w.py)
    polys, keep_polys = upload_polys(vsabi, w.polys)
    small = torch.empty(4, dtype=torch.int32, device="cuda")
    small2 = torch.empty(4, dtype=torch.int32, device="cuda")
    with pytest.raises(vsabi.CapacityError) as ei:
        vsabi.join_brute_noalloc(pts, polys, PRED_CODES["intersects"], small, small2)
    assert ei.value.required > 4
