"""vibespatial_b200: B200-native point-by-polygon spatial join.

A drop-in for ``sjoin(points, polygons, predicate='within'|'intersects')``
and ``GeometryArray.within/contains`` of vibeSpatial's GeoPandas-compatible
API.  Pairs are computed on the GPU by hand-written sm_100a kernels behind a
C-ABI (``libvsjoin.so``, declared in ``include/vsjoin.h``): an exact
point-in-polygon refine on a packed Hilbert R-tree, or on a learned cell
index with an FP32 tile-relative filter.  There is no CPU fallback.
"""
from .frame import GeoDataFrame, GeoSeries
from .geometry import (
    GeometryArray,
    GeometryDtype,
    MultiPolygon,
    Point,
    Polygon,
    box,
    points_from_xy,
)
from .io import from_wkb, geodataframe_from_arrow, geoseries_from_arrow, read_geoparquet
from .query import SpatialIndex, query_spatial_index
from .sjoin import sjoin, sjoin_nearest

__all__ = [
    "GeoDataFrame",
    "GeoSeries",
    "GeometryArray",
    "GeometryDtype",
    "MultiPolygon",
    "Point",
    "Polygon",
    "SpatialIndex",
    "box",
    "from_wkb",
    "geodataframe_from_arrow",
    "geoseries_from_arrow",
    "points_from_xy",
    "read_geoparquet",
    "query_spatial_index",
    "sjoin",
    "sjoin_nearest",
]
