"""Columnar geometry storage and the GeoPandas-compatible GeometryArray.

Storage follows the layout of the reference's OwnedGeometryArray for the
families this join handles (src/vibespatial/geometry/buffers.py:140-249,
src/vibespatial/geometry/owned.py:42-45): one tag per row (-1 null, 0 Point,
2 Polygon, 5 MultiPolygon, as in the reference's FAMILY_TAGS), point
coordinates per row, and one polygonal SoA in MultiPolygon form (a Polygon is
a one-part MultiPolygon): ``geom_off`` row -> parts, ``part_off`` part ->
rings, ``ring_off`` ring -> coordinates, ``x``/``y`` coordinates.  Empty
points have NaN coordinates; empty polygons have zero parts.

Scalars (``Point``, ``Polygon``, ``MultiPolygon``) are small immutable
value objects; Shapely is not required.
"""
from __future__ import annotations

import numbers
from dataclasses import dataclass

import numpy as np
import pandas as pd
from pandas.api.extensions import ExtensionArray, ExtensionDtype, register_extension_dtype

NULL, POINT, POLYGON, MULTIPOLYGON = -1, 0, 2, 5
_TYPE_NAMES = {POINT: "Point", POLYGON: "Polygon", MULTIPOLYGON: "MultiPolygon"}


# ----------------------------------------------------------------------------
# scalars
# ----------------------------------------------------------------------------
class BaseGeometry:
    __slots__ = ()
    geom_type = "Geometry"

    def __ne__(self, other):
        return not self == other


class Point(BaseGeometry):
    __slots__ = ("x", "y")
    geom_type = "Point"

    def __init__(self, *args):
        if len(args) == 1 and not isinstance(args[0], numbers.Number):
            args = tuple(args[0])
        if len(args) == 0:
            self.x = self.y = float("nan")
        elif len(args) == 2:
            self.x, self.y = float(args[0]), float(args[1])
        else:
            raise ValueError("Point takes (x, y) or nothing")

    @property
    def is_empty(self) -> bool:
        return bool(np.isnan(self.x) or np.isnan(self.y))

    @property
    def coords(self):
        return [] if self.is_empty else [(self.x, self.y)]

    @property
    def bounds(self):
        if self.is_empty:
            return (np.nan,) * 4
        return (self.x, self.y, self.x, self.y)

    def __eq__(self, other):
        if not isinstance(other, Point):
            return False
        if self.is_empty or other.is_empty:
            return self.is_empty and other.is_empty
        return self.x == other.x and self.y == other.y

    def __hash__(self):
        return hash(("Point", self.x, self.y))

    def __repr__(self):
        return "POINT EMPTY" if self.is_empty else f"POINT ({self.x:g} {self.y:g})"


def _ring_array(ring) -> np.ndarray:
    a = np.asarray(ring, dtype=np.float64).reshape(-1, 2)
    if len(a) and (a[0] != a[-1]).any():
        a = np.vstack([a, a[:1]])
    return a


class Polygon(BaseGeometry):
    __slots__ = ("rings",)
    geom_type = "Polygon"

    def __init__(self, shell=None, holes=None):
        if shell is None or len(shell) == 0:
            self.rings = ()
        else:
            self.rings = (_ring_array(shell),) + tuple(_ring_array(h) for h in (holes or ()))

    @classmethod
    def _from_rings(cls, rings):
        p = cls.__new__(cls)
        p.rings = tuple(rings)
        return p

    @property
    def is_empty(self) -> bool:
        return len(self.rings) == 0

    @property
    def exterior(self):
        return self.rings[0] if self.rings else np.empty((0, 2))

    @property
    def interiors(self):
        return self.rings[1:]

    @property
    def bounds(self):
        if self.is_empty:
            return (np.nan,) * 4
        a = np.vstack(self.rings)
        return (a[:, 0].min(), a[:, 1].min(), a[:, 0].max(), a[:, 1].max())

    def __eq__(self, other):
        return (isinstance(other, Polygon) and len(self.rings) == len(other.rings)
                and all(np.array_equal(a, b) for a, b in zip(self.rings, other.rings)))

    def __hash__(self):
        return hash(("Polygon", len(self.rings)))

    def __repr__(self):
        if self.is_empty:
            return "POLYGON EMPTY"
        rings = ", ".join("(" + ", ".join(f"{x:g} {y:g}" for x, y in r) + ")" for r in self.rings)
        return f"POLYGON ({rings})"


def box(minx, miny, maxx, maxy) -> Polygon:
    """Rectangle with the ring order Shapely's box() uses."""
    return Polygon([(maxx, miny), (maxx, maxy), (minx, maxy), (minx, miny)])


class MultiPolygon(BaseGeometry):
    __slots__ = ("polygons",)
    geom_type = "MultiPolygon"

    def __init__(self, polygons=None):
        polys = []
        for p in polygons or ():
            polys.append(p if isinstance(p, Polygon) else Polygon(*p) if isinstance(p, tuple) else Polygon(p))
        self.polygons = tuple(q for q in polys if not q.is_empty)

    @property
    def geoms(self):
        return self.polygons

    @property
    def is_empty(self) -> bool:
        return len(self.polygons) == 0

    @property
    def bounds(self):
        if self.is_empty:
            return (np.nan,) * 4
        b = np.array([p.bounds for p in self.polygons])
        return (b[:, 0].min(), b[:, 1].min(), b[:, 2].max(), b[:, 3].max())

    def __eq__(self, other):
        return (isinstance(other, MultiPolygon) and len(self.polygons) == len(other.polygons)
                and all(a == b for a, b in zip(self.polygons, other.polygons)))

    def __hash__(self):
        return hash(("MultiPolygon", len(self.polygons)))

    def __repr__(self):
        return "MULTIPOLYGON EMPTY" if self.is_empty else f"MULTIPOLYGON ({len(self.polygons)} parts)"


# ----------------------------------------------------------------------------
# extension dtype / array
# ----------------------------------------------------------------------------
@register_extension_dtype
class GeometryDtype(ExtensionDtype):
    name = "geometry"
    type = BaseGeometry
    kind = "O"
    na_value = None

    @classmethod
    def construct_array_type(cls):
        return GeometryArray


@dataclass(frozen=True)
class PolygonBuffers:
    x: np.ndarray
    y: np.ndarray
    ring_off: np.ndarray
    part_off: np.ndarray
    geom_off: np.ndarray
    valid: np.ndarray  # uint8 per row: 1 = polygonal and non-empty

    def __len__(self):
        return len(self.geom_off) - 1


def _ranges(starts: np.ndarray, counts: np.ndarray):
    """Concatenated index ranges [starts[k], starts[k] + counts[k]) and their offsets."""
    starts = np.asarray(starts, dtype=np.int64)
    counts = np.asarray(counts, dtype=np.int64)
    new_off = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(counts, out=new_off[1:])
    total = int(new_off[-1])
    if total == 0:
        return np.empty(0, dtype=np.int64), new_off
    idx = np.repeat(starts - new_off[:-1], counts) + np.arange(total, dtype=np.int64)
    return idx, new_off


class GeometryArray(ExtensionArray):
    """Points, Polygons and MultiPolygons in columnar form (see module docs)."""

    _dtype = GeometryDtype()

    def __init__(self, tags, px, py, geom_off, part_off, ring_off, x, y, crs=None):
        self._tags = np.asarray(tags, dtype=np.int8)
        self._px = np.asarray(px, dtype=np.float64)
        self._py = np.asarray(py, dtype=np.float64)
        self._geom_off = np.asarray(geom_off, dtype=np.int32)
        self._part_off = np.asarray(part_off, dtype=np.int32)
        self._ring_off = np.asarray(ring_off, dtype=np.int32)
        self._x = np.asarray(x, dtype=np.float64)
        self._y = np.asarray(y, dtype=np.float64)
        self.crs = crs
        n = len(self._tags)
        if not (len(self._px) == len(self._py) == n and len(self._geom_off) == n + 1):
            raise ValueError("inconsistent GeometryArray buffers")
        self._cache = {}

    # -- construction ---------------------------------------------------------
    @classmethod
    def from_points(cls, x, y, crs=None) -> "GeometryArray":
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        n = len(x)
        return cls(np.zeros(n, np.int8), x, y, np.zeros(n + 1, np.int32), np.zeros(1, np.int32),
                   np.zeros(1, np.int32), np.empty(0), np.empty(0), crs=crs)

    @classmethod
    def from_polygon_buffers(cls, x, y, ring_off, part_off, geom_off, geom_type=None, valid=None, crs=None):
        """Polygonal rows from a MultiPolygon-form SoA (tags Polygon unless a row has >1 part)."""
        geom_off = np.asarray(geom_off, dtype=np.int32)
        n = len(geom_off) - 1
        nparts = np.diff(geom_off)
        if geom_type is None:
            tags = np.where(nparts > 1, MULTIPOLYGON, POLYGON).astype(np.int8)
        else:
            gt = np.asarray(geom_type)
            tags = np.where(gt == "MultiPolygon", MULTIPOLYGON, POLYGON).astype(np.int8)
        if valid is not None:
            tags = np.where(np.asarray(valid).astype(bool), tags, NULL).astype(np.int8)
        nan = np.full(n, np.nan)
        return cls(tags, nan, nan.copy(), geom_off, part_off, ring_off, x, y, crs=crs)

    @classmethod
    def from_shapes(cls, values, crs=None) -> "GeometryArray":
        tags, px, py, xs, ys = [], [], [], [], []
        geom_off, part_off, ring_off = [0], [0], [0]
        for v in values:
            if v is None or (isinstance(v, float) and np.isnan(v)):
                tags.append(NULL)
                px.append(np.nan)
                py.append(np.nan)
                geom_off.append(geom_off[-1])
                continue
            if isinstance(v, Point):
                tags.append(POINT)
                px.append(v.x)
                py.append(v.y)
                geom_off.append(geom_off[-1])
                continue
            if isinstance(v, Polygon):
                parts = [] if v.is_empty else [v]
                tags.append(POLYGON)
            elif isinstance(v, MultiPolygon):
                parts = list(v.polygons)
                tags.append(MULTIPOLYGON)
            else:
                raise TypeError(f"unsupported geometry {type(v).__name__}")
            px.append(np.nan)
            py.append(np.nan)
            for part in parts:
                for ring in part.rings:
                    xs.append(ring[:, 0])
                    ys.append(ring[:, 1])
                    ring_off.append(ring_off[-1] + len(ring))
                part_off.append(part_off[-1] + len(part.rings))
            geom_off.append(geom_off[-1] + len(parts))
        x = np.concatenate(xs) if xs else np.empty(0)
        y = np.concatenate(ys) if ys else np.empty(0)
        return cls(np.asarray(tags, np.int8), px, py, geom_off, part_off, ring_off, x, y, crs=crs)

    @classmethod
    def _from_sequence(cls, scalars, *, dtype=None, copy=False):
        if isinstance(scalars, GeometryArray):
            return scalars.copy() if copy else scalars
        return cls.from_shapes(list(scalars))

    @classmethod
    def _from_factorized(cls, values, original):
        return cls.from_shapes(list(values))

    # -- pandas ExtensionArray protocol -----------------------------------------
    @property
    def dtype(self):
        return self._dtype

    def __len__(self) -> int:
        return len(self._tags)

    @property
    def nbytes(self) -> int:
        return int(sum(a.nbytes for a in (self._tags, self._px, self._py, self._geom_off, self._part_off,
                                          self._ring_off, self._x, self._y)))

    def isna(self):
        return self._tags == NULL

    def copy(self):
        return GeometryArray(self._tags.copy(), self._px.copy(), self._py.copy(), self._geom_off.copy(),
                             self._part_off.copy(), self._ring_off.copy(), self._x.copy(), self._y.copy(),
                             crs=self.crs)

    def _scalar(self, i):
        t = int(self._tags[i])
        if t == NULL:
            return None
        if t == POINT:
            return Point(self._px[i], self._py[i]) if not np.isnan(self._px[i]) else Point()
        polys = []
        for part in range(self._geom_off[i], self._geom_off[i + 1]):
            rings = []
            for r in range(self._part_off[part], self._part_off[part + 1]):
                a, b = self._ring_off[r], self._ring_off[r + 1]
                rings.append(np.stack([self._x[a:b], self._y[a:b]], axis=1))
            polys.append(Polygon._from_rings(rings))
        if t == POLYGON:
            return polys[0] if polys else Polygon()
        return MultiPolygon(polys)

    def __getitem__(self, item):
        if isinstance(item, (int, np.integer)):
            i = int(item)
            if i < 0:
                i += len(self)
            if not 0 <= i < len(self):
                raise IndexError(item)
            return self._scalar(i)
        if isinstance(item, slice):
            return self.take(np.arange(len(self))[item])
        item = pd.api.indexers.check_array_indexer(self, item)
        if item.dtype == bool:
            item = np.flatnonzero(item)
        return self.take(item)

    def __setitem__(self, key, value):
        raise TypeError("GeometryArray is immutable")

    def __iter__(self):
        for i in range(len(self)):
            yield self._scalar(i)

    def __array__(self, dtype=None, copy=None):
        out = np.empty(len(self), dtype=object)
        for i in range(len(self)):
            out[i] = self._scalar(i)
        return out

    def __eq__(self, other):
        if isinstance(other, GeometryArray):
            other = np.asarray(other)
        a = np.asarray(self)
        if np.ndim(other) == 0:
            return np.array([v == other for v in a], dtype=bool)
        return np.array([x == y for x, y in zip(a, other)], dtype=bool)

    def take(self, indices, allow_fill=False, fill_value=None):
        idx = np.asarray(indices, dtype=np.int64)
        if allow_fill:
            missing = idx == -1
            if (idx < -1).any():
                raise ValueError("invalid take index")
            idx = np.where(missing, 0, idx)
        else:
            missing = np.zeros(len(idx), dtype=bool)
            if len(self):
                idx = np.where(idx < 0, idx + len(self), idx)
        if len(idx) and len(self) == 0:
            if not missing.all():
                raise IndexError("take from an empty GeometryArray")
            n = len(idx)
            return GeometryArray(np.full(n, NULL, np.int8), np.full(n, np.nan), np.full(n, np.nan),
                                 np.zeros(n + 1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.int32),
                                 np.empty(0), np.empty(0), crs=self.crs)
        if len(idx) and (idx.max() >= len(self) or idx.min() < 0):
            raise IndexError("take index out of bounds")
        rows = np.where(missing, 0, idx)
        tags = self._tags[rows].copy()
        tags[missing] = NULL
        gcount = np.where(missing, 0, np.diff(self._geom_off)[rows])
        part_idx, new_geom = _ranges(self._geom_off[rows], gcount)
        ring_idx, new_part = _ranges(self._part_off[part_idx], np.diff(self._part_off)[part_idx])
        coord_idx, new_ring = _ranges(self._ring_off[ring_idx], np.diff(self._ring_off)[ring_idx])
        px = self._px[rows].copy()
        py = self._py[rows].copy()
        px[missing] = np.nan
        py[missing] = np.nan
        return GeometryArray(tags, px, py, new_geom.astype(np.int32), new_part.astype(np.int32),
                             new_ring.astype(np.int32), self._x[coord_idx], self._y[coord_idx], crs=self.crs)

    @classmethod
    def _concat_same_type(cls, to_concat):
        to_concat = list(to_concat)
        tags = np.concatenate([a._tags for a in to_concat]) if to_concat else np.empty(0, np.int8)
        px = np.concatenate([a._px for a in to_concat]) if to_concat else np.empty(0)
        py = np.concatenate([a._py for a in to_concat]) if to_concat else np.empty(0)
        geom_off, part_off, ring_off, xs, ys = [np.zeros(1, np.int64)], [np.zeros(1, np.int64)], \
            [np.zeros(1, np.int64)], [], []
        g0 = p0 = r0 = 0
        for a in to_concat:
            geom_off.append(a._geom_off[1:].astype(np.int64) + g0)
            part_off.append(a._part_off[1:].astype(np.int64) + p0)
            ring_off.append(a._ring_off[1:].astype(np.int64) + r0)
            g0 += int(a._geom_off[-1])
            p0 += int(a._part_off[-1])
            r0 += int(a._ring_off[-1])
            xs.append(a._x)
            ys.append(a._y)
        crs = to_concat[0].crs if to_concat else None
        return cls(tags, px, py, np.concatenate(geom_off), np.concatenate(part_off), np.concatenate(ring_off),
                   np.concatenate(xs) if xs else np.empty(0), np.concatenate(ys) if ys else np.empty(0), crs=crs)

    def _values_for_factorize(self):
        return np.asarray(self), None

    def __repr__(self):
        head = ", ".join(repr(self._scalar(i)) for i in range(min(len(self), 3)))
        return f"<GeometryArray [{head}{', ...' if len(self) > 3 else ''}] length {len(self)}>"

    # -- geometry helpers -------------------------------------------------------
    @property
    def geom_type(self) -> np.ndarray:
        out = np.empty(len(self), dtype=object)
        for t, name in _TYPE_NAMES.items():
            out[self._tags == t] = name
        out[self._tags == NULL] = None
        return out

    @property
    def is_empty(self) -> np.ndarray:
        pts = (self._tags == POINT) & np.isnan(self._px)
        polys = np.isin(self._tags, (POLYGON, MULTIPOLYGON)) & (np.diff(self._geom_off) == 0)
        return pts | polys

    def families(self) -> set:
        """Tags of the rows that can match anything: null and empty rows of any
        family never match (src/vibespatial/api/tools/sjoin.py:502-544), so
        they do not decide which side of a join holds the points."""
        fam = self._cache.get("families")  # the array is immutable
        if fam is None:
            live = self._tags[(self._tags != NULL) & ~self.is_empty]
            present = np.bincount(live.astype(np.int64) + 1, minlength=1)  # tags >= -1: counted, not sorted
            fam = self._cache["families"] = frozenset(int(t) - 1 for t in np.flatnonzero(present))
        return set(fam)

    def is_points(self) -> bool:
        return self.families() <= {POINT}

    def is_polygonal(self) -> bool:
        return self.families() <= {POLYGON, MULTIPOLYGON}

    def point_buffers(self):
        """(x, y, valid uint8) of a point array; null rows get valid 0."""
        valid = (self._tags == POINT).astype(np.uint8)
        return self._px, self._py, valid

    def polygon_buffers(self) -> PolygonBuffers:
        """MultiPolygon-form SoA of a polygonal array; null / empty rows never match."""
        valid = (np.isin(self._tags, (POLYGON, MULTIPOLYGON)) & (np.diff(self._geom_off) > 0)).astype(np.uint8)
        return PolygonBuffers(self._x, self._y, self._ring_off, self._part_off, self._geom_off, valid)

    @property
    def bounds(self) -> np.ndarray:
        out = np.full((len(self), 4), np.nan)
        p = self._tags == POINT
        out[p, 0] = out[p, 2] = self._px[p]
        out[p, 1] = out[p, 3] = self._py[p]
        for i in np.flatnonzero(np.isin(self._tags, (POLYGON, MULTIPOLYGON))):
            g0, g1 = self._geom_off[i], self._geom_off[i + 1]
            if g1 > g0:
                c0 = self._ring_off[self._part_off[g0]]
                c1 = self._ring_off[self._part_off[g1]]
                out[i] = (self._x[c0:c1].min(), self._y[c0:c1].min(), self._x[c0:c1].max(), self._y[c0:c1].max())
        return out

    @property
    def total_bounds(self) -> np.ndarray:
        b = self.bounds
        if np.isnan(b).all():
            return np.full(4, np.nan)
        return np.array([np.nanmin(b[:, 0]), np.nanmin(b[:, 1]), np.nanmax(b[:, 2]), np.nanmax(b[:, 3])])

    # -- element-wise predicates (point x polygon) --------------------------------
    def _binary(self, other, op: str) -> np.ndarray:
        from .predicates import binary_predicate

        return binary_predicate(self, other, op)

    def within(self, other):
        return self._binary(other, "within")

    def contains(self, other):
        return self._binary(other, "contains")

    def intersects(self, other):
        return self._binary(other, "intersects")

    def covers(self, other):
        return self._binary(other, "covers")

    def covered_by(self, other):
        return self._binary(other, "covered_by")

    def touches(self, other):
        return self._binary(other, "touches")

    def contains_properly(self, other):
        return self._binary(other, "contains_properly")

    def crosses(self, other):
        return self._binary(other, "crosses")

    def overlaps(self, other):
        return self._binary(other, "overlaps")

    def disjoint(self, other):
        return self._binary(other, "disjoint")

    def distance(self, other):
        from .predicates import distance

        return distance(self, other)

    def dwithin(self, other, distance):
        from .predicates import dwithin

        return dwithin(self, other, distance)

    # -- spatial index ----------------------------------------------------------------
    @property
    def sindex(self):
        from .query import SpatialIndex

        si = self._cache.get("sindex")
        if si is None:
            si = self._cache["sindex"] = SpatialIndex(self)
        return si


def points_from_xy(x, y, crs=None) -> GeometryArray:
    """GeoPandas' ``points_from_xy``: a point GeometryArray from coordinate arrays."""
    return GeometryArray.from_points(x, y, crs=crs)


def from_shapely_like(values, crs=None) -> GeometryArray:
    return GeometryArray.from_shapes(values, crs=crs)
