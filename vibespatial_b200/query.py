"""The operator seam of the join: ``query_spatial_index`` and ``SpatialIndex``.

Mirrors the reference's query_spatial_index(tree, flat_index, geometry, *,
predicate, sort, ...) (src/vibespatial/spatial/query.py:247-261) and the
``sindex.query`` contract it serves (src/vibespatial/api/sindex.py:144): the
result is a (2, K) intp array of (input geometry row, tree row) pairs for
which ``predicate(input geometry, tree geometry)`` holds.  Only point x
polygon combinations run here; whichever side holds the points becomes the
query side of the CUDA join, and the pairs are swapped back when the tree
holds the points (the reference swaps ``within`` <-> ``contains`` the same
way on its host path, src/vibespatial/api/tools/sjoin.py:1049-1082).
"""
from __future__ import annotations

import numpy as np

VALID_PREDICATES = {None, "intersects", "within", "contains", "contains_properly", "covers", "covered_by",
                    "touches", "overlaps", "crosses", "dwithin"}

# (points are the INPUT side) -> device predicate, or "empty" when the
# predicate can never hold between a point and a polygon
_INPUT_POINTS = {None: None, "intersects": "intersects", "within": "within", "covered_by": "covered_by",
                 "touches": "touches", "contains": "empty", "contains_properly": "empty", "covers": "empty",
                 "overlaps": "empty", "crosses": "empty"}
# (points are the TREE side)
_TREE_POINTS = {None: None, "intersects": "intersects", "contains": "within", "contains_properly": "within",
                "covers": "covered_by", "touches": "touches", "within": "empty", "covered_by": "empty",
                "overlaps": "empty", "crosses": "empty"}

# Pair generators: the CUDA joins.  Tests of the host logic substitute the
# CPU oracle here; the package itself never does.
_pairs_backend = None
_dwithin_backend = None
_nearest_backend = None
_nearest_polygons_backend = None


def _pairs(points, polygons, predicate, method, on_device=False):
    if _pairs_backend is not None:
        left, right = _pairs_backend(points, polygons, predicate)
        if on_device:
            import torch

            return (torch.from_numpy(np.asarray(left, np.int32)).cuda(),
                    torch.from_numpy(np.asarray(right, np.int32)).cuda())
        return left, right
    from ._device import join_pairs

    return join_pairs(points, polygons, predicate, method=method, on_device=on_device)


def _dwithin(points, polygons, method, on_device=False, **dist):
    """(point rows, polygon rows) within the distance (``distance``,
    ``point_distance`` or ``geom_distance``)."""
    if _dwithin_backend is not None:
        left, right = _dwithin_backend(points, polygons, **dist)
        if on_device:
            import torch

            return (torch.from_numpy(np.asarray(left, np.int32)).cuda(),
                    torch.from_numpy(np.asarray(right, np.int32)).cuda())
        return left, right
    from ._device import dwithin_pairs

    return dwithin_pairs(points, polygons, method=method, on_device=on_device, **dist)


def nearest_pairs(points, polygons, *, max_distance=None, method="learned"):
    """(point rows, polygon rows, distances): every polygon at each point's
    minimum distance, within ``max_distance`` when given, sorted by (point,
    polygon).  The query of sjoin_nearest (the reference's query_nearest with
    all ties, src/vibespatial/spatial/nearest.py)."""
    if _nearest_backend is not None:
        return _nearest_backend(points, polygons, max_distance=max_distance)
    from ._device import nearest_pairs as device_nearest

    return device_nearest(points, polygons, max_distance=max_distance, method=method)


def nearest_polygon_pairs(polygons, points, *, max_distance=None):
    """(polygon rows, point rows, distances): every point at each polygon's
    minimum distance, within ``max_distance`` when given, sorted by (polygon,
    point) -- the query of sjoin_nearest when the polygons are the matched side."""
    if _nearest_polygons_backend is not None:
        return _nearest_polygons_backend(polygons, points, max_distance=max_distance)
    from ._device import nearest_polygon_pairs as device_nearest

    return device_nearest(polygons, points, max_distance=max_distance)


def _distance_args(distance, n_geometry, geometry_is_points):
    """Per-row or scalar threshold for the join: the geometry (input) side
    owns the per-row values, whichever side holds the points."""
    if distance is None:
        raise ValueError("'distance' parameter is required for 'dwithin' predicate")
    d = np.asarray(distance, dtype=np.float64)
    if d.ndim == 0:
        return {"distance": float(d)}
    if d.shape != (n_geometry,):
        raise ValueError("Could not broadcast distance array to the number of geometries: "
                         f"{d.shape} vs ({n_geometry},)")
    return {"point_distance": d} if geometry_is_points else {"geom_distance": d}


def _query_dwithin(tree, geometry, distance, method, on_device):
    if geometry.is_points() and tree.is_polygonal():
        return _dwithin(geometry, tree, method, on_device, **_distance_args(distance, len(geometry), True))
    if geometry.is_polygonal() and tree.is_points():
        pt, poly = _dwithin(tree, geometry, method, on_device, **_distance_args(distance, len(geometry), False))
        if on_device:
            if poly.numel():
                from ._device import sort_pairs_on_device

                poly, pt = sort_pairs_on_device(poly.contiguous(), pt.contiguous())
            return poly, pt
        out = np.vstack([poly, pt]).astype(np.intp)
        order = np.lexsort((out[1], out[0]))
        return out[0][order], out[1][order]
    raise NotImplementedError(
        "vibespatial_b200 joins points with polygons/multipolygons only "
        f"(tree families {sorted(tree.families())}, input families {sorted(geometry.families())})")


def _query_device(tree, geometry, predicate, method):
    """(geometry rows, tree rows) as int32 CUDA tensors sorted by (geometry row, tree row)."""
    import torch

    empty = (torch.empty(0, dtype=torch.int32, device="cuda"), torch.empty(0, dtype=torch.int32, device="cuda"))
    if len(tree) == 0 or len(geometry) == 0:
        return empty
    if geometry.is_points() and tree.is_polygonal():
        pred = _INPUT_POINTS[predicate]
        return empty if pred == "empty" else _pairs(geometry, tree, pred, method, on_device=True)
    if geometry.is_polygonal() and tree.is_points():
        pred = _TREE_POINTS[predicate]
        if pred == "empty":
            return empty
        pt, poly = _pairs(tree, geometry, pred, method, on_device=True)
        if poly.numel():
            from ._device import sort_pairs_on_device

            poly, pt = sort_pairs_on_device(poly.contiguous(), pt.contiguous())
        return poly, pt
    raise NotImplementedError(
        "vibespatial_b200 joins points with polygons/multipolygons only "
        f"(tree families {sorted(tree.families())}, input families {sorted(geometry.families())})")


def query_spatial_index(tree, geometry, *, predicate=None, sort=False, distance=None, method="learned",
                        return_device=False):
    """(2, K) intp array of (geometry row, tree row) pairs satisfying ``predicate``.

    ``tree`` and ``geometry`` are GeometryArrays; one must hold points and the
    other polygons/multipolygons.  ``sort`` orders the pairs by (geometry row,
    tree row) (the CUDA join always returns them sorted).  ``return_device``
    returns the pairs as two int32 CUDA tensors that never leave the device
    (the reference's DeviceSpatialJoinResult, src/vibespatial/spatial/query_types.py:176).
    """
    from .geometry import GeometryArray

    if predicate not in VALID_PREDICATES:
        raise ValueError(f"Got predicate='{predicate}'; `predicate` must be one of {sorted(map(str, VALID_PREDICATES))}")
    if distance is not None and predicate != "dwithin":
        raise ValueError("'distance' parameter is only supported in combination with 'dwithin' predicate")
    if not isinstance(tree, GeometryArray) or not isinstance(geometry, GeometryArray):
        raise TypeError("query_spatial_index expects GeometryArrays")
    if predicate == "dwithin":
        if distance is None:
            raise ValueError("'distance' parameter is required for 'dwithin' predicate")
        if len(tree) == 0 or len(geometry) == 0:
            if return_device:
                import torch

                e = torch.empty(0, dtype=torch.int32, device="cuda")
                return e, e.clone()
            return np.empty((2, 0), dtype=np.intp)
        left, right = _query_dwithin(tree, geometry, distance, method, return_device)
        return (left, right) if return_device else np.vstack([left, right]).astype(np.intp)
    if return_device:
        return _query_device(tree, geometry, predicate, method)
    empty = np.empty((2, 0), dtype=np.intp)
    if len(tree) == 0 or len(geometry) == 0:
        return empty
    if geometry.is_points() and tree.is_polygonal():
        pred = _INPUT_POINTS[predicate]
        if pred == "empty":
            return empty
        left, right = _pairs(geometry, tree, pred, method)
        return np.vstack([left, right]).astype(np.intp)
    if geometry.is_polygonal() and tree.is_points():
        pred = _TREE_POINTS[predicate]
        if pred == "empty":
            return empty
        pt, poly = _pairs(tree, geometry, pred, method)
        out = np.vstack([poly, pt]).astype(np.intp)
        if out.shape[1]:
            order = np.lexsort((out[1], out[0]))
            out = out[:, order]
        return out
    raise NotImplementedError(
        "vibespatial_b200 joins points with polygons/multipolygons only "
        f"(tree families {sorted(tree.families())}, input families {sorted(geometry.families())})")


class SpatialIndex:
    """``GeometryArray.sindex``: a reusable index over the array (the tree side)."""

    valid_query_predicates = set(VALID_PREDICATES)

    def __init__(self, geometry):
        self.geometry = geometry

    def __len__(self):
        return len(self.geometry)

    @property
    def is_empty(self):
        return len(self.geometry) == 0

    @property
    def size(self):
        """Number of geometries in the index."""
        return len(self.geometry)

    def _input(self, geometry):
        """(GeometryArray, output index) of a query input."""
        import pandas as pd

        from .geometry import BaseGeometry, GeometryArray

        if isinstance(geometry, BaseGeometry):
            return GeometryArray.from_shapes([geometry]), pd.RangeIndex(1)
        index = getattr(geometry, "index", None)
        arr = getattr(geometry, "values", geometry)
        if not isinstance(arr, GeometryArray):
            arr = GeometryArray.from_shapes(list(arr))
        return arr, (index if index is not None else pd.RangeIndex(len(arr)))

    def _pair_rows(self, arr, predicate, distance):
        """(input rows, tree rows): CUDA tensors from the CUDA join, host
        arrays when a test substitutes the pair source."""
        on_device = _pairs_backend is None and _dwithin_backend is None
        res = query_spatial_index(self.geometry, arr, predicate=predicate, distance=distance,
                                  return_device=on_device)
        return res[0], res[1]

    def query_any(self, geometry, *, predicate=None, distance=None):
        """Whether each input geometry has any match (a boolean Series over
        the input's index), without exporting the pairs: the reference's
        sindex.query_any (src/vibespatial/api/sindex.py:594)."""
        import pandas as pd

        from .relation import _counts, _to_numpy

        arr, index = self._input(geometry)
        rows, _ = self._pair_rows(arr, predicate, distance)
        hit = _to_numpy(_counts(rows, len(arr))) > 0
        return pd.Series(hit, index=index)

    def query_aggregate(self, geometry, aggregations, *, predicate=None, distance=None):
        """Per input geometry, reductions over its matches without exporting
        the pairs: ``{"name": "size"}`` counts them, ``{"name": (values,
        "sum")}`` sums ``values`` (one number per tree geometry) over them;
        empty groups give 0.  The reference's sindex.query_aggregate
        (src/vibespatial/api/sindex.py:505)."""
        from collections.abc import Mapping

        import pandas as pd

        arr, index = self._input(geometry)
        n, m = len(arr), len(self.geometry)
        # validation and messages of sindex._normalize_query_aggregations and
        # _validate_query_aggregate_values (src/vibespatial/api/sindex.py:1280-1334)
        if not isinstance(aggregations, Mapping) or not aggregations:
            raise ValueError("aggregations must be a non-empty mapping")
        specs = {}
        for name, spec in aggregations.items():
            if not isinstance(name, str):
                raise TypeError("query aggregate output column names must be strings")
            if isinstance(spec, str) and spec == "size":
                specs[name] = None
                continue
            if not (isinstance(spec, tuple) and len(spec) == 2 and spec[1] == "sum"):
                raise ValueError("query aggregate specifications must be 'size' or (values, 'sum')")
            values = spec[0]
            shape = getattr(values, "shape", None)
            if shape is not None and len(shape) != 1:
                raise ValueError("query aggregate values must be one-dimensional")
            try:
                count = len(values)
            except TypeError as exc:
                raise ValueError("query aggregate values must be one-dimensional and aligned with indexed tree "
                                 "geometries") from exc
            if count != m:
                raise ValueError("query aggregate values must align with indexed tree geometries")
            raw = np.asarray(getattr(values, "to_numpy", lambda: values)())
            if not pd.api.types.is_numeric_dtype(raw.dtype):
                raise TypeError("query aggregate sum values must be numeric")
            specs[name] = raw.astype(np.float64)
        rows, trows = self._pair_rows(arr, predicate, distance)
        out = {}
        if isinstance(rows, np.ndarray):
            for name, v in specs.items():
                if v is None:
                    out[name] = np.bincount(rows, minlength=n)[:n].astype(np.int64) if len(rows) else \
                        np.zeros(n, np.int64)
                else:
                    out[name] = np.bincount(rows, weights=v[trows], minlength=n)[:n] if len(rows) else np.zeros(n)
        else:
            # the library's row-reduction kernels on the join's device pairs
            # (sorted by query row, as the sums need): vs_row_counts, vs_row_sums
            import torch

            from . import _abi

            ctx = _abi.default_context(rows.device.index if rows.device.index is not None else 0)
            for name, v in specs.items():
                if v is None:
                    out[name] = _abi.row_counts(ctx, rows, n).cpu().numpy()
                else:
                    dv = torch.from_numpy(v).to(rows.device)
                    out[name] = _abi.row_sums(ctx, rows, trows, dv, n).cpu().numpy()
        return pd.DataFrame(out, index=index)

    # -- row flow without exported pairs (the reference's private relation
    # -- methods, src/vibespatial/api/sindex.py:1592-1760, 2381) ------------

    def query_relation(self, geometry, *, predicate=None, sort=False, distance=None, return_device=True):
        """The query's pairs as a :class:`~vibespatial_b200.relation.Relation`
        (query rows on the left, indexed rows on the right, sorted by left):
        sindex.query_relation (src/vibespatial/api/sindex.py:1592).  With
        ``return_device`` (the default) the arrays are the join's CUDA tensors."""
        from .relation import Relation

        arr, _ = self._input(geometry)
        if return_device:
            rows, trows = self._pair_rows(arr, predicate, distance)
        else:
            res = query_spatial_index(self.geometry, arr, predicate=predicate, sort=sort, distance=distance)
            rows, trows = res[0], res[1]
        return Relation(rows, trows, predicate=predicate, left_row_count=len(arr),
                        right_row_count=len(self.geometry), sorted_by_left=True)

    def query_left_semijoin(self, geometry, *, predicate=None, distance=None):
        """Query rows with at least one match, ascending (a
        :class:`~vibespatial_b200.relation.RowSet`): sindex.query_left_semijoin
        (src/vibespatial/api/sindex.py:1633)."""
        return self.query_relation(geometry, predicate=predicate, distance=distance).left_semijoin_rowset()

    def query_left_antijoin(self, geometry, *, predicate=None, distance=None):
        """Query rows without any match, ascending: sindex.query_left_antijoin
        (src/vibespatial/api/sindex.py:1660)."""
        return self.query_relation(geometry, predicate=predicate, distance=distance).left_antijoin_rowset()

    def query_right_semijoin(self, geometry, *, predicate=None, distance=None):
        """Indexed rows matched by at least one query geometry, ascending:
        sindex.query_right_semijoin (src/vibespatial/api/sindex.py:1714)."""
        return self.query_relation(geometry, predicate=predicate, distance=distance).right_semijoin_rowset()

    def query_left_match_count_expression(self, geometry, *, predicate=None, distance=None):
        """Matches per query row (an int64 :class:`~vibespatial_b200.relation.Expression`):
        sindex.query_left_match_count_expression (src/vibespatial/api/sindex.py:1687)."""
        from .relation import Expression

        rel = self.query_relation(geometry, predicate=predicate, distance=distance)
        counts = rel.left_match_count_expression()
        return Expression("spatial_index.left_match_count", counts.values, source_row_count=counts.source_row_count,
                          dtype="int64")

    def query_pair_aggregate(self, other, geometry, *, predicate=None, distance=None):
        """Per indexed row position i of two aligned indexes: the query
        geometries matching ``self``'s row i (``left_count``), ``other``'s row
        i (``right_count``), and both (``shared_count``): sindex.query_pair_aggregate
        (src/vibespatial/api/sindex.py:973; shared pairs as in its host path :1257-1270)."""
        import pandas as pd

        if not isinstance(other, SpatialIndex):
            raise TypeError("other must be a SpatialIndex")
        if other.size != self.size:
            raise ValueError("query pair aggregate indexes must have equal size")
        a = self.query_relation(geometry, predicate=predicate, distance=distance)
        b = other.query_relation(geometry, predicate=predicate, distance=distance)
        m = self.size
        nq = max(int(a.left_row_count), 1)
        left = a.right_match_count_expression().to_numpy()
        right = b.right_match_count_expression().to_numpy()
        # pairs are unique, so the pairs of a also present in b are the shared ones
        if a.is_device and b.is_device:
            # membership of a's pairs among b's (b sorted by (query row, indexed
            # row), as the join returns them), then counts of the shared pairs'
            # indexed rows: vs_pairs_member, vs_row_counts
            from . import _abi

            dev = a.left_indices.device.index if a.left_indices.device.index is not None else 0
            ctx = _abi.default_context(dev)
            flags = _abi.pairs_member(ctx, a.left_indices, a.right_indices, b.left_indices, b.right_indices, nq)
            shared = _abi.row_counts(ctx, a.right_indices, m, mask=flags).cpu().numpy()
        else:
            ar, al = np.asarray(a.right_indices, np.int64), np.asarray(a.left_indices, np.int64)
            br, bl = np.asarray(b.right_indices, np.int64), np.asarray(b.left_indices, np.int64)
            both = np.isin(ar * nq + al, br * nq + bl)
            shared = np.bincount(ar[both], minlength=m)[:m] if both.any() else np.zeros(m, np.int64)
        return pd.DataFrame({"left_count": left.astype(np.int64), "right_count": right.astype(np.int64),
                             "shared_count": np.asarray(shared, np.int64)}, index=pd.RangeIndex(m))

    def nearest_relation(self, geometry, *, return_all=True, max_distance=None, exclusive=False, k=1):
        """The nearest pairs with their distances as a
        :class:`~vibespatial_b200.relation.Relation` (sindex.nearest_relation,
        src/vibespatial/api/sindex.py:2381); same arguments as :meth:`nearest`."""
        from .relation import Relation

        arr, _ = self._input(geometry)
        pairs, dist = self.nearest(arr, return_all=return_all, max_distance=max_distance, return_distance=True,
                                   exclusive=exclusive, k=k)
        return Relation(pairs[0], pairs[1], predicate="nearest", distances=dist, left_row_count=len(arr),
                        right_row_count=len(self.geometry), sorted_by_left=True)

    def intersection(self, coordinates):
        """Compatibility form of query (rtree's Index.intersection): tree rows
        whose box contains the point ``(x, y)``.  Rectangle bounds are not
        supported by this point-query join."""
        try:
            coords = tuple(coordinates)
        except TypeError as err:
            raise TypeError("Invalid coordinates, must be iterable in format (minx, miny, maxx, maxy) (for bounds) "
                            f"or (x, y) (for points). Got `coordinates` = {coordinates}.") from err
        from .geometry import Point

        if len(coords) == 2:
            return self.query(Point(*coords), predicate=None)
        if len(coords) == 4:
            raise NotImplementedError("rectangle queries are outside this point x polygon join; query a point")
        raise TypeError("Invalid coordinates, must be iterable in format (minx, miny, maxx, maxy) (for bounds) "
                        f"or (x, y) (for points). Got `coordinates` = {coordinates}.")

    def query(self, geometry, predicate=None, sort=False, distance=None, output_format="indices",
              return_device=False, method="learned"):
        """Tree rows matching ``predicate(geometry, tree geometry)``.

        ``output_format``: ``"indices"`` ((n,) tree rows for a scalar input,
        (2, n) (input row, tree row) pairs for an array), ``"sparse"`` (a
        boolean scipy.sparse COO array of shape (len(tree),) or
        (len(tree), len(geometry))), or ``"dense"`` (the same as a numpy bool
        array).  ``return_device=True`` (indices only) returns int32 CUDA
        tensors: the tree rows for a scalar input, else (input rows, tree
        rows), computed and kept on the device.  Mirrors sindex.query
        (src/vibespatial/api/sindex.py:144, output formats :463-502).
        """
        from .geometry import BaseGeometry, GeometryArray

        if output_format not in ("indices", "sparse", "dense"):
            raise ValueError(f"Invalid output_format: '{output_format}'. Use one of 'indices', 'sparse', 'dense'.")
        if return_device and output_format != "indices":
            raise ValueError("return_device=True is only supported with output_format='indices'")
        scalar = isinstance(geometry, BaseGeometry)
        if scalar:
            geometry = GeometryArray.from_shapes([geometry])
        else:
            geometry = getattr(geometry, "values", geometry)
            if not isinstance(geometry, GeometryArray):
                geometry = GeometryArray.from_shapes(list(geometry))
        if return_device:
            rows, tree_rows = query_spatial_index(self.geometry, geometry, predicate=predicate, sort=sort,
                                                  distance=distance, method=method, return_device=True)
            return tree_rows if scalar else (rows, tree_rows)
        res = query_spatial_index(self.geometry, geometry, predicate=predicate, sort=sort, distance=distance,
                                  method=method)
        n_tree = len(self.geometry)
        if output_format == "indices":
            return res[1] if scalar else res
        tree_rows, input_rows = res[1], res[0]
        if output_format == "dense":
            if scalar:
                dense = np.zeros(n_tree, dtype=bool)
                dense[tree_rows] = True
            else:
                dense = np.zeros((n_tree, len(geometry)), dtype=bool)
                dense[tree_rows, input_rows] = True
            return dense
        import scipy.sparse

        ones = np.ones(len(tree_rows), dtype=np.bool_)
        if scalar:
            return scipy.sparse.coo_array((ones, tree_rows.reshape(1, -1)), shape=(n_tree,), dtype=np.bool_)
        return scipy.sparse.coo_array((ones, (tree_rows, input_rows)), shape=(n_tree, len(geometry)),
                                      dtype=np.bool_)

    def nearest(self, geometry, return_all=True, max_distance=None, return_distance=False, exclusive=False, k=1):
        """The nearest tree geometries of every input geometry (sindex.nearest,
        src/vibespatial/api/sindex.py:2018): a (2, n) intp array of (input row,
        tree row), plus the distances with ``return_distance``.  Ties are all
        returned unless ``return_all=False`` (then the smallest tree row).
        ``max_distance`` bounds the search.  Points against polygons either way
        round; ``exclusive`` drops equal geometries, which a point and a
        polygon never are; ``k`` must be 1."""
        from .geometry import BaseGeometry, GeometryArray

        if k != 1:
            raise NotImplementedError("k-nearest (k > 1) is outside this point x polygon join")
        if max_distance is not None and max_distance < 0:
            raise ValueError("max_distance must be greater than or equal to 0")
        if isinstance(geometry, BaseGeometry):
            geometry = GeometryArray.from_shapes([geometry])
        else:
            geometry = getattr(geometry, "values", geometry)
            if not isinstance(geometry, GeometryArray):
                geometry = GeometryArray.from_shapes(list(geometry))
        tree = self.geometry
        if len(tree) == 0 or len(geometry) == 0:
            rows, trows, dist = np.empty(0, np.intp), np.empty(0, np.intp), np.empty(0, np.float64)
        elif geometry.is_points() and tree.is_polygonal():
            rows, trows, dist = nearest_pairs(geometry, tree, max_distance=max_distance)
        elif geometry.is_polygonal() and tree.is_points():
            rows, trows, dist = nearest_polygon_pairs(geometry, tree, max_distance=max_distance)
        else:
            raise NotImplementedError(
                "vibespatial_b200 joins points with polygons/multipolygons only "
                f"(tree families {sorted(tree.families())}, input families {sorted(geometry.families())})")
        rows, trows, dist = np.asarray(rows, np.intp), np.asarray(trows, np.intp), np.asarray(dist, np.float64)
        if not return_all and len(rows):
            first = np.concatenate([[True], rows[1:] != rows[:-1]])
            rows, trows, dist = rows[first], trows[first], dist[first]
        out = np.vstack([rows, trows])
        return (out, dist) if return_distance else out

