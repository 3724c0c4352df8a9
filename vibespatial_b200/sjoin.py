"""``sjoin``: the GeoPandas-compatible spatial join for points x polygons.

Drop-in for the reference's ``sjoin`` (src/vibespatial/api/tools/sjoin.py:37):
same signature, argument checks (:151-153, :268-320), predicate semantics and
output frame shape.  Pair generation runs on the GPU through
``query_spatial_index`` (the reference's seam, src/vibespatial/spatial/query.py:247);
the output frame follows the reference's relation-join export
(src/vibespatial/api/_native_results.py:301-470): index columns are reset
with ``index_<suffix>`` names, overlapping columns get suffixes, the
indexers are adjusted for ``how`` and the active geometry is the left one
(right one for ``how='right'``).  Inner-join rows are ordered by
(left row, right row).
"""
from __future__ import annotations

import warnings

import numpy as np
import pandas as pd

from .frame import GeoDataFrame
from .geometry import GeometryArray
from .query import query_spatial_index

# sjoin allows an outer join; sjoin_nearest does not (src/vibespatial/api/tools/sjoin.py:164, :294-297)
_SJOIN_HOWS = ["left", "right", "inner", "outer"]


def _maybe_make_list(obj):
    if isinstance(obj, tuple):
        return list(obj)
    if obj is not None and not isinstance(obj, list):
        return [obj]
    return obj


def _basic_checks(left_df, right_df, how, lsuffix, rsuffix, on_attribute=None, allowed_hows=None):
    if not isinstance(left_df, GeoDataFrame):
        raise ValueError(f"'left_df' should be GeoDataFrame, got {type(left_df)}")
    if not isinstance(right_df, GeoDataFrame):
        raise ValueError(f"'right_df' should be GeoDataFrame, got {type(right_df)}")
    if allowed_hows is None:
        allowed_hows = ["left", "right", "inner"]
    if how not in allowed_hows:
        raise ValueError(f'`how` was "{how}" but is expected to be in {allowed_hows}')
    lcrs, rcrs = left_df.crs, right_df.crs
    if lcrs != rcrs and lcrs is not None and rcrs is not None:
        warnings.warn(f"CRS mismatch between the CRS of left geometries and the CRS of right geometries.\n"
                      f"Left CRS: {lcrs}\nRight CRS: {rcrs}", UserWarning, stacklevel=3)
    if on_attribute:
        for attr in on_attribute:
            if attr not in left_df and attr not in right_df:
                raise ValueError(f"Expected column {attr} is missing from both of the dataframes.")
            if attr not in left_df:
                raise ValueError(f"Expected column {attr} is missing from the left dataframe.")
            if attr not in right_df:
                raise ValueError(f"Expected column {attr} is missing from the right dataframe.")
            if attr in (left_df.geometry.name, right_df.geometry.name):
                raise ValueError("Active geometry column cannot be used as an input for on_attribute parameter.")


def _geom_predicate_query(left_df, right_df, predicate, distance, method):
    """(left rows, right rows) satisfying predicate(left geometry, right
    geometry), sorted: int32 CUDA tensors from the CUDA join (they stay on the
    device for the export), host arrays when a test substitutes the pair
    source."""
    from . import query as _q

    left_geom = left_df.geometry.array
    right_geom = right_df.geometry.array
    on_device = _q._pairs_backend is None and _q._dwithin_backend is None
    # tree = right side, input = left side (the reference's STRtree orientation)
    pairs = query_spatial_index(right_geom, left_geom, predicate=predicate, sort=True, distance=distance,
                                method=method, return_device=on_device)
    return pairs[0], pairs[1]


def _attribute_codes(left_df, right_df, on_attribute):
    """int64 codes per row of each frame: equal on_attribute values, equal
    codes; a missing value anywhere gives -1 (never equal, as in pandas)."""
    nl = len(left_df)
    combined = None
    for attr in on_attribute:
        vals = pd.concat([pd.Series(left_df[attr].to_numpy()), pd.Series(right_df[attr].to_numpy())],
                         ignore_index=True)
        codes, uniq = pd.factorize(vals, use_na_sentinel=True)
        codes = codes.astype(np.int64)
        if combined is None:
            combined = codes
        else:
            miss = (combined < 0) | (codes < 0)
            mixed, _ = pd.factorize(combined * (len(uniq) + 1) + codes)
            combined = np.where(miss, -1, mixed.astype(np.int64))
    return combined[:nl], combined[nl:]


def _join_indexers(l_idx, r_idx, n_left, n_right, how, codes=None):
    """Output row indexers (-1 = missing) and each output row's source pair
    (-1 = an added row), after the on_attribute filter.  Device pairs go
    through vs_join_export; host pairs through the same steps in numpy."""
    if not isinstance(l_idx, np.ndarray):
        from ._device import export_indexers

        lc, rc = codes if codes is not None else (None, None)
        return export_indexers(l_idx, r_idx, n_left, n_right, how, lc, rc)
    l_idx = np.asarray(l_idx, np.intp)
    r_idx = np.asarray(r_idx, np.intp)
    kept = None
    if codes is not None and len(l_idx):
        lc, rc = codes
        keep = (lc[l_idx] >= 0) & (lc[l_idx] == rc[r_idx])
        kept = np.flatnonzero(keep)
        l_idx, r_idx = l_idx[keep], r_idx[keep]
    l_out, r_out, src = _adjust_indexers(l_idx, r_idx, n_left, n_right, how)
    if kept is not None:
        src = np.where(src >= 0, kept[np.maximum(src, 0)] if len(kept) else -1, -1)
    return l_out, r_out, src


def _reset_index_with_suffix(df, suffix, other):
    index_names = list(df.index.names)
    out = df.reset_index()
    cols = list(out.columns)
    for i, name in enumerate(index_names):
        if name is None:
            new = f"index_{suffix}" if len(index_names) == 1 else f"index_{suffix}{i}"
            if new in df.columns or new in other.columns:
                raise ValueError(f"'{new}' cannot be a column name in the frames being joined")
            cols[i] = new
    out.columns = pd.Index(cols)
    return out, index_names


def _suffix_overlaps(left_cols, right_cols, lsuffix, rsuffix, lgeom, rgeom):
    overlap = set(left_cols) & set(right_cols)
    if overlap and not lsuffix and not rsuffix:
        raise ValueError(f"columns overlap but no suffix specified: {sorted(map(str, overlap))}")
    left = [f"{c}_{lsuffix}" if c in overlap and c != lgeom and lsuffix is not None else c for c in left_cols]
    right = [f"{c}_{rsuffix}" if c in overlap and c != rgeom and rsuffix is not None else c for c in right_cols]
    # a suffixed name that collides with another column of the same side
    # (one that was not already repeated before renaming) is deprecated in
    # GeoPandas (src/vibespatial/api/_native_results.py:355-375)
    made = set()
    for before, after in ((left_cols, left), (right_cols, right)):
        b, a = pd.Index(before), pd.Index(after)
        made.update(a[a.duplicated() & ~b.duplicated()].tolist())
    if made:
        warnings.warn(f"Passing 'suffixes' which cause duplicate columns {made} in the result is deprecated and "
                      "will raise a MergeError in a future version.", FutureWarning, stacklevel=4)
    return left, right


def _adjust_indexers(l_idx, r_idx, n_left, n_right, how):
    """Row indexers for each ``how`` (-1 = missing row), as GeoPandas builds
    them, and for every output row the pair it came from (-1 for an added
    unmatched row)."""
    src = np.arange(len(l_idx), dtype=np.intp)
    if how == "inner":
        return l_idx, r_idx, src
    if how == "outer":
        counts = np.bincount(l_idx, minlength=n_left) if len(l_idx) else np.zeros(n_left, np.intp)
        repeats = np.maximum(counts, 1)
        out_l = np.repeat(np.arange(n_left, dtype=np.intp), repeats)
        out_r = np.full(len(out_l), -1, dtype=np.intp)
        out_src = np.full(len(out_l), -1, dtype=np.intp)
        if len(l_idx):
            starts = np.cumsum(repeats) - repeats
            rank = np.arange(len(l_idx)) - np.repeat(np.cumsum(counts) - counts, counts)
            out_r[starts[l_idx] + rank] = r_idx
            out_src[starts[l_idx] + rank] = src
        matched_right = np.zeros(n_right, dtype=bool)
        matched_right[r_idx] = True
        missing = np.flatnonzero(~matched_right)
        minus = np.full(len(missing), -1, np.intp)
        return (np.concatenate([out_l, minus]), np.concatenate([out_r, missing.astype(np.intp)]),
                np.concatenate([out_src, minus]))
    if how == "right":
        order = np.lexsort((l_idx, r_idx))
        l_idx, r_idx = r_idx[order], l_idx[order]  # swapped: the right side drives
        src = src[order]
        n = n_right
    else:
        n = n_left
    idx = np.arange(n)
    missing = idx[~np.isin(idx, l_idx)]
    ins = np.searchsorted(l_idx, missing)
    l_idx = np.insert(l_idx, ins, missing)
    r_idx = np.insert(r_idx, ins, -1)
    src = np.insert(src, ins, -1)
    if how == "right":
        l_idx, r_idx = r_idx, l_idx
    return l_idx, r_idx, src


def _take_rows(df, rows):
    """Rows by position; -1 gives an all-missing row."""
    rows = np.asarray(rows, dtype=np.intp)
    has_missing = bool((rows < 0).any())
    parts = []
    for i in range(df.shape[1]):
        col = df.iloc[:, i].reset_index(drop=True)
        arr = col.array
        if isinstance(arr, GeometryArray):
            values = arr.take(rows, allow_fill=True)
        elif has_missing:
            values = col.reindex(pd.Index(rows)).array  # -1 is not a label: missing
        else:
            values = arr.take(rows)
        parts.append(pd.Series(values, name=df.columns[i]))
    if not parts:
        return pd.DataFrame(index=pd.RangeIndex(len(rows)))
    return pd.concat(parts, axis=1)


def _frame_join(left_df, right_df, l_idx, r_idx, how, lsuffix, rsuffix, on_attribute, pair_values=None,
                value_col=None):
    """The joined frame of the (left rows, right rows) pairs; ``pair_values``
    (one float per pair, e.g. distances) becomes the last column
    ``value_col``, NaN on unmatched rows."""
    lgeom = left_df.geometry.name
    rgeom = right_df.geometry.name
    codes = _attribute_codes(left_df, right_df, on_attribute) if on_attribute else None
    if on_attribute:
        right_df = right_df.drop(columns=on_attribute)
    left = pd.DataFrame(left_df)
    right = pd.DataFrame(right_df)
    left_geometry = right_geometry = None
    if how in ("inner", "left"):
        right = right.drop(columns=[rgeom])
    elif how == "right":
        left = left.drop(columns=[lgeom])
    else:
        left_geometry = left[lgeom].array
        right_geometry = right[rgeom].array
        left = left.drop(columns=[lgeom])
        right = right.drop(columns=[rgeom])
    left_nlevels, right_nlevels = left.index.nlevels, right.index.nlevels
    left, left_names = _reset_index_with_suffix(left, lsuffix, right)
    right, right_names = _reset_index_with_suffix(right, rsuffix, left)
    lcols, rcols = _suffix_overlaps(list(left.columns), list(right.columns), lsuffix, rsuffix, lgeom, rgeom)
    left.columns, right.columns = pd.Index(lcols), pd.Index(rcols)
    left_index_cols, right_index_cols = lcols[:left_nlevels], rcols[:right_nlevels]
    l_idx, r_idx, src = _join_indexers(l_idx, r_idx, len(left), len(right), how, codes)
    lpart = _take_rows(left, l_idx)
    rpart = _take_rows(right, r_idx)
    joined = pd.concat([lpart, rpart], axis=1)
    if how in ("inner", "left"):
        joined = joined.set_index(left_index_cols)
        joined.index.names = [None if n is None else c for n, c in zip(left_names, left_index_cols)]
        geometry, crs = lgeom, left_df.crs
    elif how == "right":
        joined = joined.set_index(right_index_cols)
        joined.index.names = [None if n is None else c for n, c in zip(right_names, right_index_cols)]
        geometry, crs = rgeom, right_df.crs
    else:
        lg = left_geometry.take(l_idx, allow_fill=True)
        rg = right_geometry.take(r_idx, allow_fill=True)
        pick = np.asarray(lg.isna())
        merged = GeometryArray._concat_same_type([lg, rg]).take(
            np.where(pick, np.arange(len(lg)) + len(lg), np.arange(len(lg))))
        joined[lgeom] = pd.Series(merged, index=joined.index)
        geometry, crs = lgeom, left_df.crs
    if value_col is not None:
        vals = np.asarray(pair_values, dtype=np.float64)
        col = np.where(src >= 0, vals[np.maximum(src, 0)] if len(vals) else np.nan, np.nan)
        joined[value_col] = pd.Series(col, index=joined.index)
    return GeoDataFrame(joined, geometry=geometry, crs=crs)


def sjoin(left_df, right_df, how="inner", predicate="intersects", lsuffix="left", rsuffix="right",
          distance=None, on_attribute=None, **kwargs):
    """Spatial join of two GeoDataFrames (points with polygons/multipolygons).

    Parameters follow GeoPandas: ``how`` in {'left', 'right', 'inner',
    'outer'}; ``predicate`` one of intersects, within, contains,
    contains_properly, covers, covered_by, touches, overlaps, crosses or
    None (bounding boxes only).  ``method`` (keyword) selects the GPU index:
    'learned' (default) or 'rtree'.
    """
    method = kwargs.pop("method", "learned")
    if kwargs:
        first = next(iter(kwargs.keys()))
        raise TypeError(f"sjoin() got an unexpected keyword argument '{first}'")
    on_attribute = _maybe_make_list(on_attribute)
    _basic_checks(left_df, right_df, how, lsuffix, rsuffix, on_attribute=on_attribute, allowed_hows=_SJOIN_HOWS)
    l_idx, r_idx = _geom_predicate_query(left_df, right_df, predicate, distance, method)
    return _frame_join(left_df, right_df, l_idx, r_idx, how, lsuffix, rsuffix, on_attribute)


def sjoin_nearest(left_df, right_df, how="inner", max_distance=None, lsuffix="left", rsuffix="right",
                  distance_col=None, exclusive=False, **kwargs):
    """Nearest-neighbour join of points with polygons/multipolygons.

    Drop-in for the reference's ``sjoin_nearest``
    (src/vibespatial/api/tools/sjoin.py:1398): every row of the matched side
    (the left frame, or the right frame for ``how='right'``) gets every
    geometry of the other frame at its minimum distance (all ties), within
    ``max_distance`` when given; ``distance_col`` adds the distances.  One
    side must hold points and the other polygons: points matched to polygons
    use the polygons' index, polygons matched to points an index over the
    points.  ``exclusive`` drops equal geometries, which a point and a polygon
    never are.
    """
    from .query import nearest_pairs, nearest_polygon_pairs

    method = kwargs.pop("method", "learned")
    if kwargs:
        first = next(iter(kwargs.keys()))
        raise TypeError(f"sjoin_nearest() got an unexpected keyword argument '{first}'")
    _basic_checks(left_df, right_df, how, lsuffix, rsuffix)
    if max_distance is not None and max_distance < 0:
        raise ValueError("max_distance must be greater than or equal to 0")
    query_df, tree_df = (right_df, left_df) if how == "right" else (left_df, right_df)
    q_geom, t_geom = query_df.geometry.array, tree_df.geometry.array
    if len(q_geom) and len(t_geom) and q_geom.is_points() and t_geom.is_polygonal():
        q_rows, t_rows, dist = nearest_pairs(q_geom, t_geom, max_distance=max_distance, method=method)
    elif len(q_geom) and len(t_geom) and q_geom.is_polygonal() and t_geom.is_points():
        q_rows, t_rows, dist = nearest_polygon_pairs(q_geom, t_geom, max_distance=max_distance)
    elif len(q_geom) == 0 or len(t_geom) == 0:
        q_rows, t_rows, dist = np.empty(0, np.intp), np.empty(0, np.intp), np.empty(0, np.float64)
    else:
        raise NotImplementedError(
            "vibespatial_b200 joins points with polygons/multipolygons only "
            f"(families {sorted(q_geom.families())} and {sorted(t_geom.families())})")
    l_idx, r_idx = (t_rows, q_rows) if how == "right" else (q_rows, t_rows)
    return _frame_join(left_df, right_df, np.asarray(l_idx, np.intp), np.asarray(r_idx, np.intp), how, lsuffix,
                       rsuffix, None, pair_values=dist, value_col=distance_col)
