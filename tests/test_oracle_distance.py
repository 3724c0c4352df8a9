"""The distance oracle (oracle/distance.c) pinned on the CPU, independently of
itself: hand-computed distances, a numpy restatement of the point-segment
distance (the comp.graphics.algorithms FAQ method of GEOS's
Distance::pointToSegment; numpy rounds every operation on its own, as the
oracle compiled with -ffp-contract=off does, so the distances agree bit for
bit), and brute force over every (point, polygon) pair for the grid-indexed
dwithin, nearest and reverse nearest joins and the element-wise distance.

The oracle is the checker of the device distance joins; these tests are
what make its answers trustworthy.
"""
import math

import numpy as np
import pytest

from _shapes import SoA, box, multi, points, polygon, soa
from vibespatial_b200.testing import synthetic as syn


def _polys(oracle, p):
    return oracle.Polygons(p.x, p.y, p.ring_off, p.part_off, p.geom_off, p.valid)


def _segment_distance_np(px, py, ax, ay, bx, by):
    """Vectorised FAQ point-segment distance, one rounding per operation."""
    px, py, ax, ay, bx, by = np.broadcast_arrays(*map(np.asarray, (px, py, ax, ay, bx, by)))
    ux, uy = bx - ax, by - ay
    len2 = ux * ux + uy * uy
    with np.errstate(invalid="ignore", divide="ignore"):
        r = ((px - ax) * ux + (py - ay) * uy) / len2
        s = ((ay - py) * ux - (ax - px) * uy) / len2
        mid = np.abs(s) * np.sqrt(len2)
    da = np.sqrt((px - ax) * (px - ax) + (py - ay) * (py - ay))
    db = np.sqrt((px - bx) * (px - bx) + (py - by) * (py - by))
    degenerate = (ax == bx) & (ay == by)
    return np.where(degenerate | (r <= 0.0), da, np.where(r >= 1.0, db, mid))


def _brute_distance(oracle, P, p, px, py, g):
    """0 inside or on polygon g (the pinned exact location), else the minimum
    over its ring segments of the numpy distance; NaN for a null polygon."""
    if not p.valid[g]:
        return math.nan
    if oracle.location(px, py, P, g) != 0:
        return 0.0
    best = math.inf
    for ring in range(p.part_off[p.geom_off[g]], p.part_off[p.geom_off[g + 1]]):
        c0, c1 = p.ring_off[ring], p.ring_off[ring + 1]
        if c1 - c0 < 2:
            continue
        d = _segment_distance_np(px, py, p.x[c0:c1 - 1], p.y[c0:c1 - 1], p.x[c0 + 1:c1], p.y[c0 + 1:c1])
        best = min(best, float(d.min()))
    return best


def _envelope_distance(p, g, px, py):
    c0, c1 = p.ring_off[p.part_off[p.geom_off[g]]], p.ring_off[p.part_off[p.geom_off[g + 1]]]
    x0, x1 = p.x[c0:c1].min(), p.x[c0:c1].max()
    y0, y1 = p.y[c0:c1].min(), p.y[c0:c1].max()
    dx = x0 - px if px < x0 else (px - x1 if px > x1 else 0.0)
    dy = y0 - py if py < y0 else (py - y1 if py > y1 else 0.0)
    if dx == 0.0:
        return dy
    if dy == 0.0:
        return dx
    return math.sqrt(dx * dx + dy * dy)


def test_known_distances(oracle):
    shapes = [box(0, 0, 1, 1),
              polygon([(0, 0), (10, 0), (10, 10), (0, 10)], [[(4, 4), (6, 4), (6, 6), (4, 6)]]),
              multi(box(0, 0, 1, 1), box(5, 0, 6, 1))]
    p = soa(shapes)
    P = _polys(oracle, p)
    d = oracle.point_polygon_distance
    assert d(3.0, 0.0, P, 0) == 2.0
    assert d(2.0, 2.0, P, 0) == math.sqrt(2.0)
    assert d(0.5, -3.0, P, 0) == 3.0
    assert d(0.5, 0.5, P, 0) == 0.0  # inside
    assert d(1.0, 0.5, P, 0) == 0.0  # on the boundary
    assert d(5.0, 5.0, P, 1) == 1.0  # in the hole: distance to the hole's ring
    assert d(5.0, 4.5, P, 1) == 0.5
    assert d(3.0, 0.5, P, 2) == 2.0  # between the parts: the nearer one
    assert d(5.5, 0.5, P, 2) == 0.0


def test_nearest_ties(oracle):
    """A point equidistant from two polygons gets both; the reverse join gives
    a polygon every point at its minimum."""
    p = soa([box(0, 0, 1, 1), box(2, 0, 3, 1), box(10, 10, 11, 11)])
    P = _polys(oracle, p)
    px, py, pv = points([(1.5, 0.5), (0.5, 0.5), (4.0, 0.5), (12.0, 10.5), (10.0, 12.0)])
    l, r, d = oracle.nearest_join(px, py, pv, P)
    assert list(zip(l.tolist(), r.tolist(), d.tolist())) == [(0, 0, 0.5), (0, 1, 0.5), (1, 0, 0.0), (2, 1, 1.0),
                                                             (3, 2, 1.0), (4, 2, 1.0)]
    l, r, d = oracle.nearest_polygons_join(px, py, pv, P)
    assert list(zip(l.tolist(), r.tolist(), d.tolist())) == [(0, 1, 0.0), (1, 0, 0.5), (2, 3, 1.0), (2, 4, 1.0)]


def test_point_segment_matches_numpy_restatement(oracle):
    rng = np.random.default_rng(5)
    n = 2000
    ax, ay, bx, by, px, py = (rng.uniform(-50, 50, n) for _ in range(6))
    # degenerate segments and points on the segment's line beyond both ends
    bx[:50], by[:50] = ax[:50], ay[:50]
    t = rng.choice([-0.5, 0.0, 0.25, 1.0, 1.5], 200)
    px[50:250] = ax[50:250] + t * (bx[50:250] - ax[50:250])
    py[50:250] = ay[50:250] + t * (by[50:250] - ay[50:250])
    want = _segment_distance_np(px, py, ax, ay, bx, by)
    got = np.array([oracle.point_segment_distance(*v) for v in zip(px, py, ax, ay, bx, by)])
    np.testing.assert_array_equal(got, want)


@pytest.fixture(scope="module")
def small(oracle):
    """Star polygons with holes and multiparts, a few null polygons, points
    inside, outside, on vertices and far away, a null point and a NaN point."""
    w = syn.degenerate_join(seed=21, n_points=400, n_polys=30)
    p = w.polys
    valid = np.ones(len(p.geom_off) - 1, np.uint8)
    valid[[3, 17]] = 0
    p = SoA(p.x, p.y, p.ring_off, p.part_off, p.geom_off, valid)
    lo, hi = float(p.x.min()), float(p.x.max())
    far = np.array([[lo - 50.0, lo - 50.0], [hi + 20.0, lo], [np.nan, 0.0]])
    px = np.concatenate([w.px, far[:, 0]])
    py = np.concatenate([w.py, far[:, 1]])
    pv = np.ones(len(px), np.uint8)
    pv[7] = 0
    P = _polys(oracle, p)
    D = np.array([[_brute_distance(oracle, P, p, px[i], py[i], g) if pv[i] and not np.isnan(px[i]) else math.nan
                   for g in range(len(p.geom_off) - 1)] for i in range(len(px))])
    return p, P, px, py, pv, D


def test_point_polygon_distance_matches_brute_force(oracle, small):
    p, P, px, py, pv, D = small
    for i in range(0, len(px), 7):
        for g in range(len(p.geom_off) - 1):
            if pv[i] and p.valid[g] and not np.isnan(px[i]):
                assert oracle.point_polygon_distance(px[i], py[i], P, g) == D[i, g]


@pytest.mark.parametrize("threshold", [0.0, 0.3, 40.0, 400.0])
def test_dwithin_join_matches_brute_force(oracle, small, threshold):
    p, P, px, py, pv, D = small
    l, r, d = oracle.dwithin_join(px, py, pv, P, threshold)
    want = [(i, g) for i in range(len(px)) for g in range(len(p.geom_off) - 1)
            if not np.isnan(D[i, g]) and not (_envelope_distance(p, g, px[i], py[i]) > threshold)
            and D[i, g] <= threshold]
    assert list(zip(l.tolist(), r.tolist())) == want
    np.testing.assert_array_equal(d, [D[i, g] for i, g in want])


@pytest.mark.parametrize("max_distance", [math.inf, 1.0])
def test_nearest_join_matches_brute_force(oracle, small, max_distance):
    p, P, px, py, pv, D = small
    l, r, d = oracle.nearest_join(px, py, pv, P, max_distance)
    want = []
    for i in range(len(px)):
        row = D[i]
        if np.all(np.isnan(row)):
            continue
        m = np.nanmin(row)
        if math.isfinite(m) and m <= max_distance:
            want += [(i, g, m) for g in np.flatnonzero(row == m)]
    assert list(zip(l.tolist(), r.tolist())) == [(i, g) for i, g, _ in want]
    np.testing.assert_array_equal(d, [m for _, _, m in want])


def test_nearest_polygons_join_matches_brute_force(oracle, small):
    p, P, px, py, pv, D = small
    l, r, d = oracle.nearest_polygons_join(px, py, pv, P)
    want = []
    for g in range(len(p.geom_off) - 1):
        col = D[:, g]
        if np.all(np.isnan(col)):
            continue
        m = np.nanmin(col)
        if math.isfinite(m):
            want += [(g, i, m) for i in np.flatnonzero(col == m)]
    assert list(zip(l.tolist(), r.tolist())) == [(g, i) for g, i, _ in want]
    np.testing.assert_array_equal(d, [m for _, _, m in want])


def test_distance_aligned_matches_brute_force(oracle):
    shapes = [box(0, 0, 1, 1), None, box(2, 2, 3, 3), [], polygon([(0, 0), (4, 0), (0, 4)])]
    p = soa(shapes)
    P = _polys(oracle, p)
    px, py, pv = points([(3, 0), (0, 0), None, (1, 1), (1, 1)])
    dist, env = oracle.distance_aligned(px, py, pv, P)
    assert dist[0] == 2.0 and env[0] == 2.0
    assert np.isnan(dist[1]) and np.isnan(dist[2]) and np.isnan(dist[3])  # null polygon, null point, empty polygon
    assert dist[4] == 0.0 and env[4] == 0.0
