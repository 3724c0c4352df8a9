"""Element-wise point x polygon predicates of GeometryArray (aligned rows).

Follows the reference's point-region fast path
(src/vibespatial/predicates/binary.py:1469-1692) and its location ->
predicate mapping (src/vibespatial/predicates/point_relations.py:100-130):

=================  ===================  ====================
predicate          point left           point right
=================  ===================  ====================
within             interior             False
contains           False                interior
contains_properly  False                interior
covers             False                interior or boundary
covered_by         interior / boundary  False
intersects         interior / boundary  interior or boundary
touches            boundary             boundary
crosses, overlaps  False                False
disjoint           exterior             exterior
=================  ===================  ====================

Null and empty rows are False (the reference's NullBehavior.FALSE,
src/vibespatial/predicates/binary.py:4012-4020).
"""
from __future__ import annotations

import numpy as np

OUTSIDE, BOUNDARY, INTERIOR, MISSING = 0, 1, 2, 255

_POINT_LEFT = {
    "within": (INTERIOR,),
    "covered_by": (INTERIOR, BOUNDARY),
    "intersects": (INTERIOR, BOUNDARY),
    "touches": (BOUNDARY,),
    "contains": (),
    "contains_properly": (),
    "covers": (),
    "crosses": (),
    "overlaps": (),
    "disjoint": (OUTSIDE,),
}
_POINT_RIGHT = {
    "contains": (INTERIOR,),
    "contains_properly": (INTERIOR,),
    "covers": (INTERIOR, BOUNDARY),
    "intersects": (INTERIOR, BOUNDARY),
    "touches": (BOUNDARY,),
    "within": (),
    "covered_by": (),
    "crosses": (),
    "overlaps": (),
    "disjoint": (OUTSIDE,),
}

# Locator and distance of aligned rows: the CUDA kernels.  Tests of the host
# logic substitute the CPU oracle here; the package itself never does.
_locate_backend = None
_distance_backend = None


def _locate(points, polygons):
    if _locate_backend is not None:
        return _locate_backend(points, polygons)
    from ._device import locate_aligned

    return locate_aligned(points, polygons)


def _broadcast(other, n):
    from .geometry import BaseGeometry, GeometryArray

    if isinstance(other, GeometryArray):
        if len(other) != n:
            raise ValueError(f"Lengths of inputs do not match. Left: {n}, Right: {len(other)}")
        return other
    if isinstance(other, BaseGeometry) or other is None:
        return GeometryArray.from_shapes([other]).take(np.zeros(n, dtype=np.int64))
    return GeometryArray.from_shapes(list(other))


def binary_predicate(left, right, op: str) -> np.ndarray:
    if op not in _POINT_LEFT:
        raise ValueError(f"unsupported predicate {op!r}")
    right = _broadcast(right, len(left))
    n = len(left)
    if n == 0:
        return np.zeros(0, dtype=bool)
    if left.is_points() and right.is_polygonal():
        points, polys, table = left, right, _POINT_LEFT
    elif left.is_polygonal() and right.is_points():
        points, polys, table = right, left, _POINT_RIGHT
    else:
        raise NotImplementedError(
            "vibespatial_b200 evaluates point x polygon predicates only "
            f"(left families {sorted(left.families())}, right {sorted(right.families())})")
    accepted = table[op]
    if not accepted:
        return np.zeros(n, dtype=bool)
    loc = _locate(points, polys)
    res = np.isin(loc, accepted)
    if op == "disjoint":
        # an empty geometry is disjoint from any present geometry; a missing one from nothing
        left_na, right_na = np.asarray(left.isna()), np.asarray(right.isna())
        empty = (np.asarray(left.is_empty) & ~left_na) | (np.asarray(right.is_empty) & ~right_na)
        res |= empty & ~left_na & ~right_na
    return res


def _aligned_pair(left, right):
    right = _broadcast(right, len(left))
    if left.is_points() and right.is_polygonal():
        return left, right
    if left.is_polygonal() and right.is_points():
        return right, left
    raise NotImplementedError(
        "vibespatial_b200 evaluates point x polygon distances only "
        f"(left families {sorted(left.families())}, right {sorted(right.families())})")


def _distances(points, polygons):
    if _distance_backend is not None:
        return _distance_backend(points, polygons)
    from ._device import distance_aligned

    return distance_aligned(points, polygons)


def distance(left, right) -> np.ndarray:
    """Row-wise point-polygon distance (0 inside or on the boundary; NaN for
    null or empty rows), the distance of the reference's point-distance
    kernels (src/vibespatial/spatial/point_distance_kernels.py:238-310)."""
    n = len(left)
    if n == 0:
        return np.zeros(0, dtype=np.float64)
    points, polys = _aligned_pair(left, right)
    return _distances(points, polys)[0]


def dwithin(left, right, d) -> np.ndarray:
    """Row-wise distance(left, right) <= d, after the envelope short-circuit
    (envelope distance > d -> False); NaN distances and thresholds are False."""
    n = len(left)
    if n == 0:
        return np.zeros(0, dtype=bool)
    d = np.broadcast_to(np.asarray(d, dtype=np.float64), (n,))
    points, polys = _aligned_pair(left, right)
    dist, env = _distances(points, polys)
    with np.errstate(invalid="ignore"):
        return ~(env > d) & (dist <= d)
