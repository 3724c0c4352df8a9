"""Tiny shape builders for known-answer cases (no Shapely in this environment).

A shape is ``None`` (null row), ``[]`` (empty polygon), a polygon given as a
list of rings (each a list of (x, y); closing vertex added if missing), or
``("multi", [polygon, ...])``.
"""
from __future__ import annotations

import numpy as np


def box(minx, miny, maxx, maxy):
    # Shapely's box() ring order (counter-clockwise starting at (maxx, miny))
    return [[(maxx, miny), (maxx, maxy), (minx, maxy), (minx, miny)]]


def polygon(shell, holes=()):
    return [list(shell)] + [list(h) for h in holes]


def multi(*polys):
    return ("multi", list(polys))


class SoA:
    def __init__(self, x, y, ring_off, part_off, geom_off, valid):
        self.x, self.y = np.asarray(x, float), np.asarray(y, float)
        self.ring_off = np.asarray(ring_off, np.int32)
        self.part_off = np.asarray(part_off, np.int32)
        self.geom_off = np.asarray(geom_off, np.int32)
        self.valid = np.asarray(valid, np.uint8)

    def __len__(self):
        return len(self.geom_off) - 1


def soa(shapes) -> SoA:
    xs, ys, ring_off, part_off, geom_off, valid = [], [], [0], [0], [0], []
    for s in shapes:
        if s is None:
            parts, v = [], 0
        elif isinstance(s, tuple) and s[0] == "multi":
            parts, v = s[1], 1
        elif len(s) == 0:
            parts, v = [], 1
        else:
            parts, v = [s], 1
        for part in parts:
            for ring in part:
                r = [tuple(map(float, p)) for p in ring]
                if r[0] != r[-1]:
                    r.append(r[0])
                xs.extend(p[0] for p in r)
                ys.extend(p[1] for p in r)
                ring_off.append(ring_off[-1] + len(r))
            part_off.append(part_off[-1] + len(part))
        geom_off.append(geom_off[-1] + len(parts))
        valid.append(v)
    return SoA(xs, ys, ring_off, part_off, geom_off, valid)


def points(pts):
    """None -> null row; () -> empty point (NaN); (x, y) -> point."""
    px, py, pv = [], [], []
    for p in pts:
        if p is None:
            px.append(np.nan); py.append(np.nan); pv.append(0)
        elif len(p) == 0:
            px.append(np.nan); py.append(np.nan); pv.append(1)
        else:
            px.append(float(p[0])); py.append(float(p[1])); pv.append(1)
    return np.asarray(px), np.asarray(py), np.asarray(pv, np.uint8)


# ---------------------------------------------------------------------------
# Known-answer cases from the reference test-suite (expected = polygon.covers(point)
# as in src/vibespatial/testing/oracle.py:276-289; None = null row).
# ---------------------------------------------------------------------------
def _short_edge_point():
    mid = np.asarray([0.0001, 0.00005])
    nrm = np.asarray([-0.0001, 0.0002])
    nrm /= np.linalg.norm(nrm)
    p = mid + nrm * 1e-5
    return (float(p[0]), float(p[1]))


KNOWN_COVERS = {
    # tests/test_point_in_polygon.py:52-70
    "boxes_empties_nulls": (
        [box(0, 0, 2, 2), [], None, box(5, 1, 9, 3), polygon([(0, 0), (4, 0), (4, 4), (0, 4)])],
        [None, (), (1, 1), (8, 2), (4, 2)],
        [None, False, None, True, True],
    ),
    # tests/test_point_in_polygon.py:73-89
    "multipolygon": (
        [multi(box(0, 0, 2, 2)[0:1], box(10, 10, 12, 12)), multi(box(0, 0, 2, 2)), multi()],
        [(1, 1), (3, 3), (0, 0)],
        [True, False, False],
    ),
    # tests/test_point_in_polygon.py:116-132 (holes, multipart)
    "holes_multipart": (
        [box(0, 0, 2, 2), multi(box(5, 5, 8, 8), box(10, 10, 12, 12)),
         polygon([(0, 0), (4, 0), (4, 4), (0, 4)], holes=[[(1, 1), (3, 1), (3, 3), (1, 3), (1, 1)]]), multi()],
        [(1, 1), (11, 11), (2, 2), (0, 0)],
        [True, True, False, False],
    ),
    # tests/test_point_in_polygon.py:135-162 (a point one microdegree outside a diagonal edge)
    "fp32_trap": (
        [polygon([(-113.0, 35.0), (-110.0, 37.0), (-110.0, 35.0), (-113.0, 35.0)])] * 3,
        [(-111.5000005547002, 36.0000008320503), (-179.0, -80.0), (179.0, 80.0)],
        [False, False, False],
    ),
    # tests/test_point_in_polygon.py:165-190 (short edge, point 1e-5 outside)
    "short_edge": (
        [polygon([(0.0, 0.0), (0.0002, 0.0001), (0.0002, -0.0001), (0.0, 0.0)])],
        [_short_edge_point()],
        [False],
    ),
}

# tests/test_spatial_query.py:2787-2848: tree boxes x query points, predicate intersects
SPATIAL_QUERY_CASE = (
    [box(0, 0, 5, 5), box(3, 3, 6, 6), box(10, 10, 11, 11)],
    [(1, 1), (4, 4), (20, 20)],
    ([0, 1, 1], [0, 0, 1]),
)
