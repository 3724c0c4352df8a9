"""Pin the exact CPU oracle before trusting it (CPU only).

* orientation sign vs exact rational arithmetic (fractions.Fraction)
* the reference test-suite's known answers for this path:
  - NYBB boroughs x 21 grid points (tests/upstream/geopandas/tools/tests/test_sjoin.py:839-898)
  - Natural Earth cities x countries, 213 rows (same file :1039-1044)
  - point-in-polygon unit cases (tests/test_point_in_polygon.py:52-190)
  - tree-box query pairs (tests/test_spatial_query.py:2787-2848)
"""
import json
import random
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

import _shapes as S

GOLDEN = Path(__file__).resolve().parent / "golden"


def _exact_sign(ax, ay, bx, by, cx, cy):
    d = (Fraction(ax) - Fraction(cx)) * (Fraction(by) - Fraction(cy)) - (Fraction(ay) - Fraction(cy)) * (Fraction(bx) - Fraction(cx))
    return (d > 0) - (d < 0)


def test_orient2d_matches_rationals(oracle):
    rng = random.Random(7)
    for t in range(20000):
        k = t % 4
        if k == 0:
            v = [rng.uniform(-1e3, 1e3) for _ in range(6)]
        elif k == 1:  # nearly collinear, UTM magnitudes
            ax, ay, bx, by = (rng.uniform(5e5, 6e5) for _ in range(4))
            s = rng.random()
            cx, cy = ax + s * (bx - ax), ay + s * (by - ay)
            if rng.random() < 0.5:
                cx = float(np.nextafter(cx, np.inf if rng.random() < 0.5 else -np.inf))
            v = [ax, ay, bx, by, cx, cy]
        elif k == 2:  # tiny edge at a large offset
            ax, ay = 3e6 + rng.uniform(-1, 1) * 1e-3, 3e6 + rng.uniform(-1, 1) * 1e-3
            bx, by = ax + rng.choice([1, -1]) * 2.0 ** -20, ay + 2.0 ** -21
            v = [ax, ay, bx, by, ax + (bx - ax) * 0.5, ay + (by - ay) * 0.5]
        else:  # mixed magnitudes
            v = [rng.uniform(-1, 1) * rng.choice([1e-10, 1.0, 1e10, 3e6]) for _ in range(6)]
        assert oracle.orient2d(*v) == _exact_sign(*v), v


def test_orient2d_exact_zero_and_ulp(oracle):
    # exactly collinear dyadic points and their one-ulp neighbours
    a, b = (0.0, 0.0), (1024.0, 512.0)
    for k in range(1, 1024, 37):
        t = k / 1024.0
        c = (a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1]))
        assert oracle.orient2d(*a, *b, *c) == 0
        up = (c[0], float(np.nextafter(c[1], np.inf)))
        dn = (c[0], float(np.nextafter(c[1], -np.inf)))
        assert oracle.orient2d(*a, *b, *up) == 1
        assert oracle.orient2d(*a, *b, *dn) == -1


@pytest.mark.parametrize("name", sorted(S.KNOWN_COVERS))
def test_known_point_in_polygon_cases(oracle, name):
    polys, pts, expected = S.KNOWN_COVERS[name]
    P = S.soa(polys)
    px, py, pv = S.points(pts)
    loc = oracle.locate_aligned(px, py, pv, oracle.Polygons(P.x, P.y, P.ring_off, P.part_off, P.geom_off, P.valid))
    got = [bool(v in (1, 2)) if v != 255 else None for v in loc]
    exp = [e if e is not None else None for e in expected]
    # 255 covers both null (None) and empty (False) rows
    for g, e, p, poly in zip(got, exp, pts, polys):
        if g is None:
            assert e in (None, False)
        else:
            assert g == e, (name, p)


def test_spatial_query_tree_boxes(oracle):
    tree, pts, (el, er) = S.SPATIAL_QUERY_CASE
    P = S.soa(tree)
    px, py, _ = S.points(pts)
    l, r = oracle.join(px, py, None, oracle.Polygons(P.x, P.y, P.ring_off, P.part_off, P.geom_off), "intersects")
    assert l.tolist() == el and r.tolist() == er


def _load(name):
    return dict(np.load(GOLDEN / name, allow_pickle=False))


def nybb_points(d, oracle):
    P = oracle.Polygons(d["x"], d["y"], d["ring_off"], d["part_off"], d["geom_off"])
    b = P.bounds()
    tb = [int(b[:, 0].min()), int(b[:, 1].min()), int(b[:, 2].max()), int(b[:, 3].max())]
    n = 20
    xs = list(range(tb[0], tb[2], int((tb[2] - tb[0]) / n)))
    ys = list(range(tb[1], tb[3], int((tb[3] - tb[1]) / n)))
    pts = list(zip(xs, ys))
    return P, np.array([p[0] for p in pts], float), np.array([p[1] for p in pts], float)


def test_nybb_known_answers(oracle):
    exp = json.loads((GOLDEN / "expected.json").read_text())
    d = _load("nybb.npz")
    P, px, py = nybb_points(d, oracle)
    assert len(px) == exp["nybb_within_left_shape"]["value"][0]
    lw, rw = oracle.join(px, py, None, P, "within")
    li, ri = oracle.join(px, py, None, P, "intersects")
    # inner join rows = matched pairs; left join rows = pairs + unmatched points
    assert len(li) == exp["nybb_inner_intersects_shape"]["value"][0]
    left_rows = len(lw) + (len(px) - len(np.unique(lw)))
    assert left_rows == exp["nybb_within_left_shape"]["value"][0]
    row1 = rw[lw == 1]
    assert len(row1) == 1 and d["attr_BoroName"][row1[0]] == exp["nybb_within_left_row1_boro"]["value"]
    right_rows = len(li) + (len(d["geom_off"]) - 1 - len(np.unique(ri)))
    assert right_rows == exp["nybb_right_intersects_shape"]["value"][0]


def test_natural_earth_cities_countries(oracle):
    exp = json.loads((GOLDEN / "expected.json").read_text())
    w = _load("naturalearth_lowres.npz")
    c = _load("naturalearth_cities.npz")
    P = oracle.Polygons(w["x"], w["y"], w["ring_off"], w["part_off"], w["geom_off"])
    l, r = oracle.join(c["x"], c["y"], None, P, "intersects")
    assert len(l) == exp["cities_countries_inner_intersects_shape"]["value"][0]


def test_oracle_join_matches_bruteforce_locations(oracle):
    """The oracle's grid join equals per-pair location over all pairs (small case)."""
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=11, n_points=3000, n_polys=60)
    P = oracle.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    l, r = oracle.join(w.px, w.py, None, P, "intersects")
    exp = []
    for i in range(len(w.px)):
        for g in range(len(P)):
            if oracle.location(w.px[i], w.py[i], P, g) != oracle.OUTSIDE:
                exp.append((i, g))
    assert list(zip(l.tolist(), r.tolist())) == exp
