"""GeoArrow and GeoParquet ingest into GeometryArrays, without Shapely.

Mirrors the reference's Arrow entry points for the families the join reads:

- ``geoseries_from_arrow`` / ``geodataframe_from_arrow``
  (src/vibespatial/io/geoarrow.py:2630-2672);
- ``read_geoparquet`` (src/vibespatial/io/geoparquet.py:3430);
- ``from_wkb`` (``decode_wkb_arrow_array_owned``, src/vibespatial/io/wkb.py:5224).

Native GeoArrow encodings (``geoarrow.point`` separated or interleaved,
``geoarrow.polygon``, ``geoarrow.multipolygon``) are read zero-copy from the
Arrow buffers: their offsets already are the MultiPolygon-form SoA the join
consumes.  WKB columns (``geoarrow.wkb``, GeoParquet's default encoding) are
decoded on the GPU by ``vs_wkb_plan_create/decode`` (``csrc/wkb.cu``).
Other families raise NotImplementedError.
"""
from __future__ import annotations

import json

import numpy as np

from .geometry import MULTIPOLYGON, NULL, POINT, POLYGON, GeometryArray

_NATIVE = ("geoarrow.point", "geoarrow.polygon", "geoarrow.multipolygon")


def _pa():
    import pyarrow as pa

    return pa


def _extension_name(field) -> str | None:
    md = field.metadata or {}
    name = md.get(b"ARROW:extension:name")
    if name is not None:
        return name.decode()
    t = getattr(field, "type", None)
    ext = getattr(t, "extension_name", None)
    return ext


def _combine(arr):
    pa = _pa()
    if isinstance(arr, pa.ChunkedArray):
        arr = arr.combine_chunks() if arr.num_chunks != 1 else arr.chunk(0)
    if isinstance(arr, pa.ExtensionArray):
        arr = arr.storage
    return arr


def _list_level(a):
    """(offsets rebased to 0, the child values they address) of a list array."""
    o = np.asarray(a.offsets.to_numpy(zero_copy_only=False), dtype=np.int64)
    child = a.values.slice(int(o[0]), int(o[-1] - o[0]))
    return o - o[0], child


def _coords(a):
    """x, y of a GeoArrow coordinate array (struct<x, y, ...> or fixed_size_list<double>[d])."""
    pa = _pa()
    if pa.types.is_struct(a.type):
        fields = a.flatten()
        names = [a.type.field(i).name for i in range(a.type.num_fields)]
        x = fields[names.index("x")].to_numpy(zero_copy_only=False)
        y = fields[names.index("y")].to_numpy(zero_copy_only=False)
        return np.asarray(x, np.float64), np.asarray(y, np.float64)
    if pa.types.is_fixed_size_list(a.type):
        d = a.type.list_size
        flat = np.asarray(a.flatten().to_numpy(zero_copy_only=False), np.float64).reshape(-1, d)
        return np.ascontiguousarray(flat[:, 0]), np.ascontiguousarray(flat[:, 1])
    raise TypeError(f"not a GeoArrow coordinate array: {a.type}")


def _native(arr, kind: str, crs=None) -> GeometryArray:
    n = len(arr)
    valid = np.asarray(arr.is_valid().to_numpy(zero_copy_only=False), dtype=bool)
    if kind == "geoarrow.point":
        x, y = _coords(arr)
        tags = np.where(valid, POINT, NULL).astype(np.int8)
        return GeometryArray(tags, np.where(valid, x, np.nan), np.where(valid, y, np.nan),
                             np.zeros(n + 1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.int32),
                             np.empty(0), np.empty(0), crs=crs)
    if kind == "geoarrow.polygon":
        o_rings, rings = _list_level(arr)          # row -> rings
        o_coords, coords = _list_level(rings)      # ring -> coordinates
        # an empty polygon owns no part; a null row keeps whatever rings Arrow
        # stores for it (its tag makes it never match)
        has = np.diff(o_rings) > 0
        geom_off = np.concatenate([[0], np.cumsum(has)])
        part_off = np.append(o_rings[:-1][has], o_rings[-1])
        tags = np.where(valid, POLYGON, NULL).astype(np.int8)
    elif kind == "geoarrow.multipolygon":
        o_parts, parts = _list_level(arr)          # row -> parts
        o_rings, rings = _list_level(parts)        # part -> rings
        o_coords, coords = _list_level(rings)      # ring -> coordinates
        geom_off = o_parts
        part_off = o_rings
        tags = np.where(valid, MULTIPOLYGON, NULL).astype(np.int8)
    else:
        raise NotImplementedError(f"GeoArrow encoding {kind!r} is outside the point/polygon join")
    x, y = _coords(coords)
    nan = np.full(n, np.nan)
    return GeometryArray(tags, nan, nan.copy(), geom_off.astype(np.int32), np.asarray(part_off, np.int32),
                         np.asarray(o_coords, np.int32), x, y, crs=crs)


def from_wkb(values, *, crs=None, on_invalid: str = "raise", device: int = 0) -> GeometryArray:
    """GeometryArray from WKB values (an Arrow binary array or a sequence of bytes/None), decoded on the GPU.

    ``on_invalid``: ``"raise"`` (ValueError on malformed WKB,
    NotImplementedError on other geometry types) or ``"ignore"`` (such rows
    become nulls).
    """
    import torch

    from . import _abi

    if on_invalid not in ("raise", "ignore"):
        raise ValueError("on_invalid must be 'raise' or 'ignore'")
    pa = _pa()
    if isinstance(values, (pa.Array, pa.ChunkedArray)):
        a = _combine(values)
        if not (pa.types.is_binary(a.type) or pa.types.is_large_binary(a.type)):
            raise TypeError(f"WKB values must be binary, got {a.type}")
        _, obuf, dbuf = a.buffers()
        odt = np.int64 if pa.types.is_large_binary(a.type) else np.int32
        o = np.frombuffer(obuf, dtype=odt)[a.offset:a.offset + len(a) + 1].astype(np.int64)
        data = (np.frombuffer(dbuf, dtype=np.uint8)[o[0]:o[-1]].copy() if dbuf is not None and len(a)
                else np.empty(0, np.uint8))
        offsets = o - o[0]
        valid = np.asarray(a.is_valid().to_numpy(zero_copy_only=False), dtype=np.uint8)
    else:
        vals = list(values)
        lens = np.array([0 if v is None else len(v) for v in vals], dtype=np.int64)
        offsets = np.concatenate([[0], np.cumsum(lens)])
        data = np.frombuffer(b"".join(v for v in vals if v is not None), dtype=np.uint8).copy()
        valid = np.array([v is not None for v in vals], dtype=np.uint8)
    n = len(offsets) - 1
    if not torch.cuda.is_available():
        raise RuntimeError("WKB decode needs a CUDA device; there is no CPU path")
    dev = torch.device("cuda", device)
    d_data = torch.from_numpy(np.ascontiguousarray(data)).to(dev) if len(data) else torch.zeros(1, dtype=torch.uint8,
                                                                                                 device=dev)
    d_off = torch.from_numpy(np.ascontiguousarray(offsets)).to(dev)
    d_valid = torch.from_numpy(valid).to(dev) if n else None
    sizes, out = _abi.wkb_decode(_abi.default_context(device), d_data, d_off, d_valid)
    if on_invalid == "raise":
        if sizes["n_malformed"]:
            raise ValueError(f"{sizes['n_malformed']} of {n} WKB values are malformed")
        if sizes["n_unsupported"]:
            raise NotImplementedError(f"{sizes['n_unsupported']} WKB values are not Point/Polygon/MultiPolygon")
    host = {k: v.cpu().numpy() for k, v in out.items()}
    ga = GeometryArray(host["tags"], host["px"], host["py"], host["geom_off"], host["part_off"], host["ring_off"],
                       host["x"], host["y"], crs=crs)
    return ga


def geometry_array_from_arrow(arr, *, field=None, crs=None, on_invalid: str = "raise") -> GeometryArray:
    """GeometryArray from an Arrow geometry column: native GeoArrow or WKB."""
    pa = _pa()
    kind = _extension_name(field) if field is not None else None
    if kind is None and isinstance(arr, pa.ExtensionArray):
        kind = arr.type.extension_name
    a = _combine(arr)
    if kind in _NATIVE:
        return _native(a, kind, crs=crs)
    if kind in (None, "geoarrow.wkb", "ogc.wkb") and (pa.types.is_binary(a.type) or pa.types.is_large_binary(a.type)):
        return from_wkb(a, crs=crs, on_invalid=on_invalid)
    raise NotImplementedError(f"Arrow geometry column of type {a.type} ({kind}) is outside the point/polygon join")


def geoseries_from_arrow(arr, **kwargs):
    """GeoSeries from an Arrow geometry array (geoarrow.* extension or WKB binary)."""
    from .frame import GeoSeries

    field = kwargs.pop("field", None)
    crs = kwargs.pop("crs", None)
    return GeoSeries(geometry_array_from_arrow(arr, field=field, crs=crs), crs=crs, **kwargs)


def _geo_columns(table, geometry=None):
    """{column: (encoding, crs)} from GeoParquet 'geo' metadata or geoarrow field metadata."""
    md = table.schema.metadata or {}
    cols = {}
    if b"geo" in md:
        geo = json.loads(md[b"geo"])
        for name, spec in geo.get("columns", {}).items():
            cols[name] = (spec.get("encoding", "WKB"), spec.get("crs"))
        primary = geo.get("primary_column")
    else:
        primary = None
        for f in table.schema:
            kind = _extension_name(f)
            if kind and kind.startswith("geoarrow."):
                cols[f.name] = (kind, None)
    if geometry is not None:
        primary = geometry
    if primary is None and cols:
        primary = next(iter(cols))
    return cols, primary


def geodataframe_from_arrow(table, *, geometry=None, to_pandas_kwargs=None, on_invalid: str = "raise"):
    """GeoDataFrame from an Arrow table whose geometry columns are GeoArrow or WKB (GeoParquet metadata)."""
    from .frame import GeoDataFrame, GeoSeries

    cols, primary = _geo_columns(table, geometry)
    if primary is None or primary not in table.column_names:
        raise ValueError("no geometry column found (no GeoParquet 'geo' metadata and no geoarrow.* field)")
    plain = [c for c in table.column_names if c not in cols]
    df = table.select(plain).to_pandas(**(to_pandas_kwargs or {}))
    for name in table.column_names:
        if name not in cols:
            continue
        enc, crs = cols[name]
        field = table.schema.field(name)
        kind = {"point": "geoarrow.point", "polygon": "geoarrow.polygon",
                "multipolygon": "geoarrow.multipolygon"}.get(str(enc).lower(), _extension_name(field))
        ga = (_native(_combine(table.column(name)), kind, crs=crs) if kind in _NATIVE
              else geometry_array_from_arrow(table.column(name), field=field, crs=crs, on_invalid=on_invalid))
        df[name] = GeoSeries(ga, index=df.index, crs=crs)
    df = df[table.column_names]
    return GeoDataFrame(df, geometry=primary, crs=cols[primary][1])


def _row_bounds(ga: GeometryArray) -> np.ndarray:
    """(n, 4) bounds, vectorised over the coordinate arrays (NaN for null/empty rows)."""
    n = len(ga)
    out = np.full((n, 4), np.nan)
    p = ga._tags == POINT
    out[p, 0] = out[p, 2] = ga._px[p]
    out[p, 1] = out[p, 3] = ga._py[p]
    if len(ga._x):
        # coordinate -> row through the offsets
        ring_row = np.repeat(np.arange(len(ga._part_off) - 1), np.diff(ga._part_off))
        part_row = np.repeat(np.arange(n), np.diff(ga._geom_off))
        coord_ring = np.repeat(np.arange(len(ga._ring_off) - 1), np.diff(ga._ring_off))
        row = part_row[ring_row[coord_ring]]
        for k, (arr, fn) in enumerate(((ga._x, np.fmin), (ga._y, np.fmin), (ga._x, np.fmax), (ga._y, np.fmax))):
            acc = np.full(n, np.inf if fn is np.fmin else -np.inf)
            fn.at(acc, row, arr)
            has = np.diff(ga._geom_off) > 0
            out[has, k] = acc[has]
    return out


def read_geoparquet(path, *, columns=None, bbox=None, to_pandas_kwargs=None, on_invalid: str = "raise", **kwargs):
    """Read a GeoParquet file into a GeoDataFrame (pyarrow reads, WKB decodes on the GPU).

    ``bbox = (minx, miny, maxx, maxy)`` keeps the rows whose geometry bounds
    intersect it.
    """
    import pyarrow.parquet as pq

    table = pq.read_table(path, columns=columns, **kwargs)
    gdf = geodataframe_from_arrow(table, to_pandas_kwargs=to_pandas_kwargs, on_invalid=on_invalid)
    if bbox is not None:
        b = _row_bounds(gdf.geometry.values)
        minx, miny, maxx, maxy = bbox
        keep = (b[:, 0] <= maxx) & (b[:, 2] >= minx) & (b[:, 1] <= maxy) & (b[:, 3] >= miny)
        gdf = gdf[keep]
    return gdf
