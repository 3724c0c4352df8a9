"""ctypes wrapper around the exact CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: this module is the checker that the CUDA join is
compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import it; the product package never does.

The C source (``oracle/exact_pip.c``) restates, with an exact orientation
predicate, the reference's point location:

* ring classification  -- src/vibespatial/cuda/device_functions/point_in_ring.py:148-188
* polygon/multipolygon -- src/vibespatial/predicates/point_relations_kernels.py:37-96
* predicate mapping    -- src/vibespatial/predicates/point_relations.py:100-130

``oracle/distance.c`` restates the distance joins (dwithin with the
reference's distance <= threshold refine, src/vibespatial/spatial/nearest.py:2855
and point_distance_kernels.py:238-310; nearest with all ties) by brute force.

``oracle/wkb.c`` restates the reference's staged WKB decode
(src/vibespatial/io/wkb.py:3755-3781 header scan, :3954 and :4043 payload
walks) as the checker of the device WKB decoder.

Parity pins: ``tests/test_oracle_golden.py`` checks this oracle against the
reference test-suite's known answers (NYBB boroughs, Natural Earth
cities x countries, the point-in-polygon unit cases) and against exact
rational arithmetic (``fractions.Fraction``) for the orientation predicate.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
_lib = None

OUTSIDE, BOUNDARY, INTERIOR = 0, 1, 2

# location -> accepted?  bit k set means location k satisfies the predicate
# (point on the left / query side, polygon on the right / tree side).
ACCEPT_MASKS = {
    None: 0,
    "intersects": (1 << BOUNDARY) | (1 << INTERIOR),
    "within": 1 << INTERIOR,
    "covered_by": (1 << BOUNDARY) | (1 << INTERIOR),
    "touches": 1 << BOUNDARY,
}

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> Path:
    """Compile ``liboracle.so`` with the committed Makefile."""
    srcs = [_HERE / "exact_pip.c", _HERE / "wkb.c", _HERE / "distance.c"]
    if force or not _LIB_PATH.exists() or any(_LIB_PATH.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(_HERE), "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        L.orc_orient2d.restype = ctypes.c_int
        L.orc_orient2d.argtypes = [ctypes.c_double] * 6
        L.orc_geometry_location.restype = ctypes.c_int
        L.orc_geometry_location.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _i32p, _i32p, _i32p, ctypes.c_int64]
        L.orc_locate_aligned.restype = None
        L.orc_locate_aligned.argtypes = [_dp, _dp, _u8p, ctypes.c_int64, _dp, _dp, _i32p, _i32p, _i32p, _u8p, _u8p, ctypes.c_int]
        L.orc_join.restype = ctypes.c_void_p
        L.orc_join.argtypes = [_dp, _dp, _u8p, ctypes.c_int64, _dp, _dp, _i32p, _i32p, _i32p, _u8p, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        L.orc_pairs_count.restype = ctypes.c_int64
        L.orc_pairs_count.argtypes = [ctypes.c_void_p]
        L.orc_pairs_copy.restype = None
        L.orc_pairs_copy.argtypes = [ctypes.c_void_p, _i32p, _i32p]
        L.orc_pairs_free.restype = None
        L.orc_pairs_free.argtypes = [ctypes.c_void_p]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_geometry_bounds.restype = None
        L.orc_geometry_bounds.argtypes = [_dp, _dp, _i32p, _i32p, _i32p, _u8p, ctypes.c_int64, _dp]
        _i64p = ctypes.POINTER(ctypes.c_int64)
        L.orc_wkb_count.restype = None
        L.orc_wkb_count.argtypes = [_u8p, _i64p, _u8p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int8), _dp, _dp,
                                    _i64p, _i64p, ctypes.c_int]
        L.orc_wkb_fill.restype = None
        L.orc_wkb_fill.argtypes = [_u8p, _i64p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int8), _i64p, _i32p, _i32p,
                                   _i32p, _dp, _dp, ctypes.c_int]
        L.orc_point_segment_distance.restype = ctypes.c_double
        L.orc_point_segment_distance.argtypes = [ctypes.c_double] * 6
        L.orc_point_polygon_distance.restype = ctypes.c_double
        L.orc_point_polygon_distance.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _i32p, _i32p, _i32p,
                                                 ctypes.c_int64]
        L.orc_dwithin_join.restype = ctypes.c_void_p
        L.orc_dwithin_join.argtypes = [_dp, _dp, _u8p, ctypes.c_int64, _dp, _dp, _i32p, _i32p, _i32p, _u8p,
                                       ctypes.c_int64, _dp, _dp, ctypes.c_double, ctypes.c_int]
        L.orc_nearest_join.restype = ctypes.c_void_p
        L.orc_nearest_join.argtypes = [_dp, _dp, _u8p, ctypes.c_int64, _dp, _dp, _i32p, _i32p, _i32p, _u8p,
                                       ctypes.c_int64, ctypes.c_double, ctypes.c_int]
        L.orc_distance_aligned.restype = None
        L.orc_distance_aligned.argtypes = [_dp, _dp, _u8p, ctypes.c_int64, _dp, _dp, _i32p, _i32p, _i32p, _u8p, _dp,
                                           _dp]
        L.orc_nearest_polygons_join.restype = ctypes.c_void_p
        L.orc_nearest_polygons_join.argtypes = [_dp, _dp, _u8p, ctypes.c_int64, _dp, _dp, _i32p, _i32p, _i32p, _u8p,
                                                ctypes.c_int64, ctypes.c_double, ctypes.c_int]
        L.orc_dpairs_count.restype = ctypes.c_int64
        L.orc_dpairs_count.argtypes = [ctypes.c_void_p]
        L.orc_dpairs_copy.restype = None
        L.orc_dpairs_copy.argtypes = [ctypes.c_void_p, _i32p, _i32p, _dp]
        L.orc_dpairs_free.restype = None
        L.orc_dpairs_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


def orient2d(ax, ay, bx, by, cx, cy) -> int:
    """Exact sign of (ax-cx)(by-cy) - (ay-cy)(bx-cx)."""
    return int(lib().orc_orient2d(ax, ay, bx, by, cx, cy))


class Polygons:
    """Polygon/multipolygon SoA: geom_off -> parts, part_off -> rings, ring_off -> coords."""

    def __init__(self, x, y, ring_off, part_off, geom_off, valid=None):
        self.x = _f64(x)
        self.y = _f64(y)
        self.ring_off = _i32(ring_off)
        self.part_off = _i32(part_off)
        self.geom_off = _i32(geom_off)
        self.valid = _u8(valid)

    def __len__(self):
        return len(self.geom_off) - 1

    def args(self):
        return (_p(self.x, _dp), _p(self.y, _dp), _p(self.ring_off, _i32p),
                _p(self.part_off, _i32p), _p(self.geom_off, _i32p))

    def bounds(self) -> np.ndarray:
        out = np.empty((len(self), 4), dtype=np.float64)
        lib().orc_geometry_bounds(*self.args(), _p(self.valid, _u8p), len(self), _p(out, _dp))
        return out


def location(px: float, py: float, polys: Polygons, g: int) -> int:
    return int(lib().orc_geometry_location(float(px), float(py), *polys.args(), int(g)))


def locate_aligned(px, py, pvalid, polys: Polygons, threads: int = 0) -> np.ndarray:
    """Row-wise location codes (0/1/2; 255 where either side is null or empty)."""
    px, py, pvalid = _f64(px), _f64(py), _u8(pvalid)
    n = len(px)
    assert len(polys) == n
    out = np.empty(n, dtype=np.uint8)
    lib().orc_locate_aligned(_p(px, _dp), _p(py, _dp), _p(pvalid, _u8p), n, *polys.args(),
                             _p(polys.valid, _u8p), _p(out, _u8p), int(threads))
    return out


def join(px, py, pvalid, polys: Polygons, predicate="within", threads: int = 0):
    """Sorted (left=point row, right=polygon row) pairs satisfying ``predicate``."""
    px, py, pvalid = _f64(px), _f64(py), _u8(pvalid)
    mask = ACCEPT_MASKS[predicate] if not isinstance(predicate, int) else int(predicate)
    L = lib()
    h = L.orc_join(_p(px, _dp), _p(py, _dp), _p(pvalid, _u8p), len(px), *polys.args(),
                   _p(polys.valid, _u8p), len(polys), mask, int(threads))
    try:
        n = L.orc_pairs_count(h)
        left = np.empty(n, dtype=np.int32)
        right = np.empty(n, dtype=np.int32)
        if n:
            L.orc_pairs_copy(h, _p(left, _i32p), _p(right, _i32p))
    finally:
        L.orc_pairs_free(h)
    return left, right


WKB_SIZE_KEYS = ("n_rows", "n_points", "n_polygons", "n_multipolygons", "n_null", "n_unsupported", "n_malformed",
                 "n_parts", "n_rings", "n_coords")


def wkb_decode(data, offsets, valid=None, threads: int = 0):
    """Decode WKB rows (Arrow binary layout: bytes + n + 1 int64 offsets).

    Returns (sizes dict, dict of numpy arrays tags, px, py, geom_off,
    part_off, ring_off, x, y) -- the device decoder's layout.
    """
    data = np.ascontiguousarray(data, dtype=np.uint8)
    if data.size == 0:
        data = np.zeros(1, np.uint8)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    valid = _u8(valid)
    n = len(off) - 1
    threads = int(threads) or nthreads_default()
    i64p = ctypes.POINTER(ctypes.c_int64)
    i8p = ctypes.POINTER(ctypes.c_int8)
    out = dict(tags=np.empty(n, np.int8), px=np.empty(n, np.float64), py=np.empty(n, np.float64))
    counts = np.empty(max(3 * n, 1), np.int64)
    sizes = np.zeros(10, np.int64)
    L = lib()
    L.orc_wkb_count(_p(data, _u8p), _p(off, i64p), _p(valid, _u8p), n, _p(out["tags"], i8p), _p(out["px"], _dp),
                    _p(out["py"], _dp), _p(counts, i64p), _p(sizes, i64p), threads)
    sz = dict(zip(WKB_SIZE_KEYS, (int(v) for v in sizes)))
    out["geom_off"] = np.empty(n + 1, np.int32)
    out["part_off"] = np.empty(sz["n_parts"] + 1, np.int32)
    out["ring_off"] = np.empty(sz["n_rings"] + 1, np.int32)
    out["x"] = np.empty(sz["n_coords"], np.float64)
    out["y"] = np.empty(sz["n_coords"], np.float64)
    L.orc_wkb_fill(_p(data, _u8p), _p(off, i64p), n, _p(out["tags"], i8p), _p(counts, i64p),
                   _p(out["geom_off"], _i32p), _p(out["part_off"], _i32p), _p(out["ring_off"], _i32p),
                   _p(out["x"], _dp), _p(out["y"], _dp), threads)
    return sz, out


def _dpairs(h):
    L = lib()
    try:
        n = L.orc_dpairs_count(h)
        left = np.empty(n, dtype=np.int32)
        right = np.empty(n, dtype=np.int32)
        dist = np.empty(n, dtype=np.float64)
        if n:
            L.orc_dpairs_copy(h, _p(left, _i32p), _p(right, _i32p), _p(dist, _dp))
    finally:
        L.orc_dpairs_free(h)
    return left, right, dist


def point_segment_distance(px: float, py: float, ax: float, ay: float, bx: float, by: float) -> float:
    """Distance from (px, py) to the segment (ax, ay)-(bx, by)."""
    return float(lib().orc_point_segment_distance(float(px), float(py), float(ax), float(ay), float(bx), float(by)))


def point_polygon_distance(px: float, py: float, polys: Polygons, g: int) -> float:
    return float(lib().orc_point_polygon_distance(float(px), float(py), *polys.args(), int(g)))


def dwithin_join(px, py, pvalid, polys: Polygons, distance=0.0, *, point_distance=None, geom_distance=None,
                 threads: int = 0):
    """Sorted (point row, polygon row, distance) with distance <= the threshold
    (per point, per polygon or the scalar ``distance``)."""
    px, py, pvalid = _f64(px), _f64(py), _u8(pvalid)
    dp = None if point_distance is None else _f64(point_distance)
    dg = None if geom_distance is None else _f64(geom_distance)
    h = lib().orc_dwithin_join(_p(px, _dp), _p(py, _dp), _p(pvalid, _u8p), len(px), *polys.args(),
                               _p(polys.valid, _u8p), len(polys), _p(dp, _dp), _p(dg, _dp), float(distance),
                               int(threads))
    return _dpairs(h)


def nearest_join(px, py, pvalid, polys: Polygons, max_distance=float("inf"), threads: int = 0):
    """Sorted (point row, polygon row, distance): every polygon at each point's
    minimum distance when that minimum is finite and <= max_distance."""
    px, py, pvalid = _f64(px), _f64(py), _u8(pvalid)
    h = lib().orc_nearest_join(_p(px, _dp), _p(py, _dp), _p(pvalid, _u8p), len(px), *polys.args(),
                               _p(polys.valid, _u8p), len(polys), float(max_distance), int(threads))
    return _dpairs(h)


def distance_aligned(px, py, pvalid, polys: Polygons):
    """Row-wise (distance, envelope distance) of point i and polygon i; NaN for null / empty rows."""
    px, py, pvalid = _f64(px), _f64(py), _u8(pvalid)
    n = len(px)
    assert len(polys) == n
    dist = np.empty(n, np.float64)
    env = np.empty(n, np.float64)
    lib().orc_distance_aligned(_p(px, _dp), _p(py, _dp), _p(pvalid, _u8p), n, *polys.args(), _p(polys.valid, _u8p),
                               _p(dist, _dp), _p(env, _dp))
    return dist, env


def nearest_polygons_join(px, py, pvalid, polys: Polygons, max_distance=float("inf"), threads: int = 0):
    """Sorted (polygon row, point row, distance): every point at each polygon's
    minimum distance when that minimum is finite and <= max_distance."""
    px, py, pvalid = _f64(px), _f64(py), _u8(pvalid)
    h = lib().orc_nearest_polygons_join(_p(px, _dp), _p(py, _dp), _p(pvalid, _u8p), len(px), *polys.args(),
                                        _p(polys.valid, _u8p), len(polys), float(max_distance), int(threads))
    return _dpairs(h)


def max_threads() -> int:
    return int(lib().orc_max_threads())


def nthreads_default() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", "0")) or max_threads()
