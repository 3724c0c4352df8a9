"""GeoSeries / GeoDataFrame: pandas containers with an active geometry column.

Only the surface the point-in-polygon join needs is provided: construction,
the active ``geometry`` column, ``set_geometry``, ``crs``, ``total_bounds``,
the element-wise ``within`` / ``contains`` / ``intersects`` / ``covers`` /
``covered_by`` / ``touches`` (reference: GeoSeries.within/contains,
src/vibespatial/api/geo_base.py:4461/3314) and ``GeoDataFrame.sjoin``
(src/vibespatial/api/geodataframe.py:6848).
"""
from __future__ import annotations

import pandas as pd

from .geometry import BaseGeometry, GeometryArray, GeometryDtype


def _to_geometry_array(data, crs=None):
    if isinstance(data, GeometryArray):
        return data
    if isinstance(data, pd.Series) and isinstance(data.dtype, GeometryDtype):
        return data.array
    return GeometryArray.from_shapes(list(data), crs=crs)


class GeoSeries(pd.Series):
    """A pandas Series backed by a GeometryArray."""

    def __init__(self, data=None, index=None, crs=None, name=None, copy=None, **kwargs):
        if data is not None and not isinstance(data, (pd.Series, GeometryArray)) or (
                isinstance(data, pd.Series) and not isinstance(data.dtype, GeometryDtype)):
            if isinstance(data, pd.Series):
                index = data.index if index is None else index
                name = data.name if name is None else name
                data = list(data)
            data = GeometryArray.from_shapes(list(data) if data is not None else [], crs=crs)
        elif data is None:
            data = GeometryArray.from_shapes([], crs=crs)
        super().__init__(data, index=index, name=name, copy=copy, **kwargs)
        if crs is not None and isinstance(self.array, GeometryArray):
            self.array.crs = crs

    @property
    def _constructor(self):
        return _geoseries_or_series

    @property
    def _constructor_expanddim(self):
        return GeoDataFrame

    @property
    def crs(self):
        return getattr(self.array, "crs", None)

    @property
    def geom_type(self):
        return pd.Series(self.array.geom_type, index=self.index)

    @property
    def is_empty(self):
        return pd.Series(self.array.is_empty, index=self.index)

    @property
    def bounds(self):
        return pd.DataFrame(self.array.bounds, columns=["minx", "miny", "maxx", "maxy"], index=self.index)

    @property
    def total_bounds(self):
        return self.array.total_bounds

    @property
    def sindex(self):
        return self.array.sindex

    def _rowwise(self, other, fn, align):
        if isinstance(other, GeoSeries):
            if align is None or align:
                this, other = self.align(other)
                this_arr, other_arr = this.array, other.array
                index = this.index
            else:
                this_arr, other_arr, index = self.array, other.array, self.index
            return pd.Series(fn(this_arr, other_arr), index=index)
        if isinstance(other, BaseGeometry):
            return pd.Series(fn(self.array, other), index=self.index)
        return pd.Series(fn(self.array, _to_geometry_array(other)), index=self.index)

    def _binary(self, other, op, align):
        return self._rowwise(other, lambda a, b: a._binary(b, op), align)

    def distance(self, other, align=None):
        """Row-wise distance to ``other`` (point x polygon rows)."""
        return self._rowwise(other, lambda a, b: a.distance(b), align)

    def dwithin(self, other, distance, align=None):
        """Row-wise ``distance(self, other) <= distance`` (point x polygon rows)."""
        return self._rowwise(other, lambda a, b: a.dwithin(b, distance), align)

    def within(self, other, align=None):
        return self._binary(other, "within", align)

    def contains(self, other, align=None):
        return self._binary(other, "contains", align)

    def intersects(self, other, align=None):
        return self._binary(other, "intersects", align)

    def covers(self, other, align=None):
        return self._binary(other, "covers", align)

    def covered_by(self, other, align=None):
        return self._binary(other, "covered_by", align)

    def touches(self, other, align=None):
        return self._binary(other, "touches", align)

    def contains_properly(self, other, align=None):
        return self._binary(other, "contains_properly", align)

    def crosses(self, other, align=None):
        return self._binary(other, "crosses", align)

    def overlaps(self, other, align=None):
        return self._binary(other, "overlaps", align)

    def disjoint(self, other, align=None):
        return self._binary(other, "disjoint", align)


def _geoseries_or_series(*args, **kwargs):
    s = pd.Series(*args, **kwargs)
    if isinstance(s.dtype, GeometryDtype):
        return GeoSeries(s.array, index=s.index, name=s.name)
    return s


class GeoDataFrame(pd.DataFrame):
    """A pandas DataFrame with an active geometry column."""

    _metadata = ["_geometry_column_name"]
    _geometry_column_name = None

    def __init__(self, data=None, *args, geometry=None, crs=None, **kwargs):
        super().__init__(data, *args, **kwargs)
        if geometry is None and isinstance(data, GeoDataFrame):
            geometry = data._geometry_column_name
        if geometry is None and "geometry" in self.columns:
            geometry = "geometry"
        if geometry is None:
            return
        if isinstance(geometry, str):
            if geometry not in self.columns:
                raise ValueError(f"geometry column {geometry!r} not found")
            col = geometry
        else:
            col = "geometry"
            values = _to_geometry_array(geometry, crs=crs)
            if len(self.columns) == 0 and len(self) == 0 and len(values):
                # no data columns: the frame takes the geometry's rows (and its index, for a series)
                index = getattr(geometry, "index", None)
                index = index if isinstance(index, pd.Index) and len(index) == len(values) else \
                    pd.RangeIndex(len(values))
                self[col] = pd.Series(values, index=index)
            else:
                if len(values) != len(self):
                    raise ValueError("geometry length does not match the frame")
                self[col] = pd.Series(values, index=self.index)
        if not isinstance(self[col].dtype, GeometryDtype):
            self[col] = pd.Series(_to_geometry_array(self[col], crs=crs), index=self.index)
        if crs is not None:
            self[col].array.crs = crs
        object.__setattr__(self, "_geometry_column_name", col)

    @property
    def _constructor(self):
        return _geodataframe_or_dataframe

    def _constructor_from_mgr(self, mgr, axes):
        df = pd.DataFrame._from_mgr(mgr, axes=axes)
        return _geodataframe_or_dataframe(df, geometry_column=self._geometry_column_name)

    @property
    def _constructor_sliced(self):
        return _geoseries_or_series

    def _constructor_sliced_from_mgr(self, mgr, axes):
        s = pd.Series._from_mgr(mgr, axes)
        s._name = None
        return _geoseries_or_series(s)

    @property
    def geometry(self) -> GeoSeries:
        name = self._geometry_column_name
        if name is None or name not in self.columns:
            raise AttributeError("No active geometry column (set one with set_geometry)")
        col = self[name]
        return col if isinstance(col, GeoSeries) else GeoSeries(col.array, index=self.index, name=name)

    def set_geometry(self, col, crs=None):
        out = self.copy()
        if isinstance(col, str):
            if not isinstance(out[col].dtype, GeometryDtype):
                out[col] = pd.Series(_to_geometry_array(out[col], crs=crs), index=out.index)
            object.__setattr__(out, "_geometry_column_name", col)
            return out
        out["geometry"] = pd.Series(_to_geometry_array(col, crs=crs), index=out.index)
        object.__setattr__(out, "_geometry_column_name", "geometry")
        return out

    def rename_geometry(self, col):
        out = self.rename(columns={self._geometry_column_name: col})
        object.__setattr__(out, "_geometry_column_name", col)
        return out

    @property
    def crs(self):
        try:
            return self.geometry.crs
        except AttributeError:
            return None

    @property
    def total_bounds(self):
        return self.geometry.total_bounds

    @property
    def sindex(self):
        return self.geometry.sindex

    def sjoin(self, df, how="inner", predicate="intersects", lsuffix="left", rsuffix="right", **kwargs):
        from .sjoin import sjoin

        return sjoin(self, df, how=how, predicate=predicate, lsuffix=lsuffix, rsuffix=rsuffix, **kwargs)

    def sjoin_nearest(self, right, how="inner", max_distance=None, lsuffix="left", rsuffix="right",
                      distance_col=None, exclusive=False, **kwargs):
        from .sjoin import sjoin_nearest

        return sjoin_nearest(self, right, how=how, max_distance=max_distance, lsuffix=lsuffix, rsuffix=rsuffix,
                             distance_col=distance_col, exclusive=exclusive, **kwargs)


def _geodataframe_or_dataframe(*args, geometry_column=None, **kwargs):
    df = pd.DataFrame(*args, **kwargs)
    geo_cols = [c for c in df.columns if isinstance(df[c].dtype, GeometryDtype)] if df.columns.is_unique else []
    if not geo_cols:
        return df
    name = geometry_column if geometry_column in geo_cols else ("geometry" if "geometry" in geo_cols else geo_cols[0])
    out = GeoDataFrame(df, geometry=name)
    return out
