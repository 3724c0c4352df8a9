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


@pytest.mark.parametrize("predicate", ["within", "intersects", "touches", None])
def test_noalloc_null_empty_and_nan_rows(vsabi, ctx, predicate):
    """Null and empty polygons, a polygon with one NaN vertex, null points and NaN points: the same pairs as
    vs_join (brute), whose index builder also spans a box over the finite coordinates only."""
    import torch
    from types import SimpleNamespace

    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=23, n_points=30_000, n_polys=400)
    p = w.polys
    x, y = p.x.copy(), p.y.copy()
    x[p.ring_off[p.part_off[p.geom_off[5]]] + 2] = np.nan  # one NaN vertex in polygon 5
    m = len(p.geom_off) - 1
    # three empty polygon rows (no parts) appended, and every ninth row null
    geom_off = np.concatenate([p.geom_off, np.full(3, p.geom_off[-1], np.int32)])
    gvalid = (np.arange(m + 3) % 9 != 4).astype(np.uint8)
    polys = SimpleNamespace(x=x, y=y, ring_off=p.ring_off, part_off=p.part_off, geom_off=geom_off, valid=gvalid)
    px, py = w.px.copy(), w.py.copy()
    px[::13] = np.nan
    py[::17] = np.nan
    pvalid = (np.arange(len(px)) % 7 != 3).astype(np.uint8)
    el, er, _ = gpu_join(vsabi, ctx, px, py, polys, predicate, method=2, pvalid=pvalid)
    pts, keep_pts = upload_points(vsabi, px, py, pvalid)
    dpolys, keep_polys = upload_polys(vsabi, polys)
    cap = len(el) + 16
    for _ in range(2):
        left = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        right = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        n = vsabi.join_brute_noalloc(pts, dpolys, PRED_CODES[predicate], left, right)
        gl, gr = _sorted_pairs(left[:n].cpu().numpy(), right[:n].cpu().numpy())
        assert n == len(el)
        np.testing.assert_array_equal(gl, el)
        np.testing.assert_array_equal(gr, er)
    assert not np.isin(er, np.flatnonzero(gvalid == 0)).any()


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
