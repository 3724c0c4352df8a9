"""Host <-> device bridge between GeometryArrays and the C-ABI library.

GeometryArray buffers are uploaded once and cached on the array (the
reference does the same with its owned device state, ``move_to``:
src/vibespatial/geometry/owned.py).  The polygon side's index is built once
per array and per method and reused by later joins, as the reference caches
its flat index on the tree array (``owned_flat_sindex``,
src/vibespatial/api/tools/sjoin.py:566-571).

There is no CPU fallback: every entry point raises when no CUDA device or no
built library is available.
"""
from __future__ import annotations

import numpy as np

from . import _abi

PREDICATE_CODES = {
    None: _abi.PRED_BBOX,
    "intersects": _abi.PRED_INTERSECTS,
    "within": _abi.PRED_WITHIN,
    "covered_by": _abi.PRED_COVERED_BY,
    "touches": _abi.PRED_TOUCHES,
}


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("vibespatial_b200 needs a CUDA device (B200); none is visible and there is no CPU path")
    return torch


def _dev(a, torch, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def device_points(ga, device: int = 0):
    """(vs_points struct, keep-alive tensors) for a point GeometryArray."""
    cached = ga._cache.get(("dpoints", device))
    if cached is None:
        torch = _torch()
        x, y, valid = ga.point_buffers()
        t = dict(x=_dev(x, torch, device), y=_dev(y, torch, device), valid=_dev(valid, torch, device))
        cached = (_abi.make_points(t["x"], t["y"], t["valid"]), t)
        ga._cache[("dpoints", device)] = cached
    return cached


def device_polygons(ga, device: int = 0):
    cached = ga._cache.get(("dpolys", device))
    if cached is None:
        torch = _torch()
        pb = ga.polygon_buffers()
        t = dict(x=_dev(pb.x, torch, device), y=_dev(pb.y, torch, device),
                 ring_off=_dev(pb.ring_off, torch, device), part_off=_dev(pb.part_off, torch, device),
                 geom_off=_dev(pb.geom_off, torch, device), valid=_dev(pb.valid, torch, device))
        cached = (_abi.make_polygons(t["x"], t["y"], t["ring_off"], t["part_off"], t["geom_off"], t["valid"]), t)
        ga._cache[("dpolys", device)] = cached
    return cached


def polygon_index(ga, learned: bool = True, device: int = 0) -> "_abi.DeviceIndex":
    key = ("index", device, learned)
    idx = ga._cache.get(key)
    if idx is None:
        ctx = _abi.default_context(device)
        P, _ = device_polygons(ga, device)
        idx = ga._cache[key] = _abi.DeviceIndex(ctx, P, learned=learned)
    return idx


def join_pairs(points, polygons, predicate, *, method: str = "learned", device: int = 0,
               on_device: bool = False):
    """Sorted (point row, polygon row) pairs satisfying ``predicate`` (point on the left).

    Host intp arrays, or with ``on_device`` the int32 CUDA tensors the join
    wrote (no device-to-host copy).
    """
    code = PREDICATE_CODES[predicate]
    if len(points) == 0 or len(polygons) == 0:
        if on_device:
            torch = _torch()
            e = torch.empty(0, dtype=torch.int32, device=device)
            return e, e.clone()
        return np.empty(0, np.intp), np.empty(0, np.intp)
    learned = method == "learned"
    index = polygon_index(polygons, learned=learned, device=device)
    pts, _ = device_points(points, device)
    m = _abi.METHOD_LEARNED if learned else (_abi.METHOD_BRUTE if method == "brute" else _abi.METHOD_RTREE)
    left, right, _ = index.join(pts, code, m, sort=True)
    if on_device:
        return left, right
    return left.cpu().numpy().astype(np.intp), right.cpu().numpy().astype(np.intp)


def sort_pairs_on_device(left, right, device: int = 0):
    """Sort int32 device pairs by (left, right) in place (in-house radix sort)."""
    _abi.sort_pairs(_abi.default_context(device), left, right)
    return left, right


def locate_aligned(points, polygons, device: int = 0) -> np.ndarray:
    """Row-wise location codes 0 outside / 1 boundary / 2 interior / 255 null-or-empty."""
    torch = _torch()
    n = len(points)
    if n == 0:
        return np.empty(0, np.uint8)
    ctx = _abi.default_context(device)
    pts, _ = device_points(points, device)
    P, _ = device_polygons(polygons, device)
    out = torch.empty(n, dtype=torch.uint8, device=device)
    _abi.locate_aligned(ctx, pts, P, out)
    return out.cpu().numpy()


def dwithin_pairs(points, polygons, *, distance=None, point_distance=None, geom_distance=None, method="learned",
                  device: int = 0, on_device: bool = False):
    """Sorted (point row, polygon row) pairs with distance(point, polygon) <= the
    threshold: ``point_distance`` (one per point), ``geom_distance`` (one per
    polygon) or the scalar ``distance``."""
    if len(points) == 0 or len(polygons) == 0:
        if on_device:
            torch = _torch()
            e = torch.empty(0, dtype=torch.int32, device=device)
            return e, e.clone()
        return np.empty(0, np.intp), np.empty(0, np.intp)
    torch = _torch()
    index = polygon_index(polygons, learned=method == "learned", device=device)
    pts, _ = device_points(points, device)
    pd_ = None if point_distance is None else _dev(np.asarray(point_distance, np.float64), torch, device)
    gd_ = None if geom_distance is None else _dev(np.asarray(geom_distance, np.float64), torch, device)
    left, right, _ = index.dwithin(pts, distance=0.0 if distance is None else float(distance), point_distance=pd_,
                                   geom_distance=gd_, sort=True)
    if on_device:
        return left, right
    return left.cpu().numpy().astype(np.intp), right.cpu().numpy().astype(np.intp)


def nearest_pairs(points, polygons, *, max_distance=None, method="learned", device: int = 0):
    """Sorted (point row, polygon row, distance): every polygon at each point's
    minimum distance (within ``max_distance`` when given)."""
    if len(points) == 0 or len(polygons) == 0:
        return np.empty(0, np.intp), np.empty(0, np.intp), np.empty(0, np.float64)
    index = polygon_index(polygons, learned=method == "learned", device=device)
    pts, _ = device_points(points, device)
    md = float("inf") if max_distance is None else float(max_distance)
    left, right, dist, _ = index.nearest(pts, max_distance=md, sort=True)
    return (left.cpu().numpy().astype(np.intp), right.cpu().numpy().astype(np.intp),
            dist.cpu().numpy())


def export_indexers(left, right, n_left: int, n_right: int, how: str, left_code=None, right_code=None,
                    device: int = 0):
    """Join export on the device (vs_join_export): host intp arrays (left
    rows, right rows, source pair) after the attribute filter and ``how``."""
    torch = _torch()
    ctx = _abi.default_context(device)
    lc = None if left_code is None else _dev(np.asarray(left_code, np.int64), torch, device)
    rc = None if right_code is None else _dev(np.asarray(right_code, np.int64), torch, device)
    out_l, out_r, src = _abi.join_export(ctx, left.contiguous(), right.contiguous(), n_left, n_right, how, lc, rc)
    return (out_l.cpu().numpy().astype(np.intp), out_r.cpu().numpy().astype(np.intp),
            src.cpu().numpy().astype(np.intp))


def distance_aligned(points, polygons, device: int = 0):
    """Row-wise (distance, envelope distance) float64 arrays; NaN for null or empty rows."""
    torch = _torch()
    n = len(points)
    if n == 0:
        return np.empty(0, np.float64), np.empty(0, np.float64)
    ctx = _abi.default_context(device)
    pts, _ = device_points(points, device)
    P, _ = device_polygons(polygons, device)
    dist = torch.empty(n, dtype=torch.float64, device=device)
    env = torch.empty(n, dtype=torch.float64, device=device)
    _abi.distance_aligned(ctx, pts, P, dist, env)
    return dist.cpu().numpy(), env.cpu().numpy()


def point_index(points, device: int = 0) -> "_abi.DeviceIndex":
    """The points' index for nearest-point queries, built once per array."""
    key = ("pindex", device)
    idx = points._cache.get(key)
    if idx is None:
        _torch()
        _, t = device_points(points, device)
        idx = points._cache[key] = _abi.point_index(_abi.default_context(device), t["x"], t["y"], t["valid"])
    return idx


def nearest_polygon_pairs(polygons, points, *, max_distance=None, device: int = 0):
    """Sorted (polygon row, point row, distance): every point at each polygon's
    minimum distance (within ``max_distance`` when given)."""
    if len(points) == 0 or len(polygons) == 0:
        return np.empty(0, np.intp), np.empty(0, np.intp), np.empty(0, np.float64)
    ctx = _abi.default_context(device)
    pidx = point_index(points, device)
    P, _ = device_polygons(polygons, device)
    md = float("inf") if max_distance is None else float(max_distance)
    left, right, dist, _ = _abi.nearest_polygons(ctx, pidx, P, max_distance=md)
    return (left.cpu().numpy().astype(np.intp), right.cpu().numpy().astype(np.intp), dist.cpu().numpy())
