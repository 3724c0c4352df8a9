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
}
_POINT_RIGHT = {
    "contains": (INTERIOR,),
    "contains_properly": (INTERIOR,),
    "covers": (INTERIOR, BOUNDARY),
    "intersects": (INTERIOR, BOUNDARY),
    "touches": (BOUNDARY,),
    "within": (),
    "covered_by": (),
}

# Locator used for aligned rows: the CUDA kernel.  Tests of the host logic
# substitute the CPU oracle here; the package itself never does.
_locate_backend = None


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
    return np.isin(loc, accepted)
