"""GeoArrow / GeoParquet ingest: native encodings (CPU), WKB decoded on the GPU,
and joins of ingested columns against the oracle."""
import json

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

import _wkb as W
import vibespatial_b200 as vs
from vibespatial_b200 import io as vio

PT = pa.struct([("x", pa.float64()), ("y", pa.float64())])


def _ring(cx, cy, r, n=6):
    a = np.linspace(0, 2 * np.pi, n, endpoint=False)
    ring = np.c_[cx + r * np.cos(a), cy + r * np.sin(a)]
    return np.vstack([ring, ring[:1]])


def _shapes():
    hole = _ring(5, 5, 0.5)[::-1]
    return [vs.Polygon(_ring(0, 0, 1)), None, vs.Polygon(_ring(5, 5, 2), [hole]),
            vs.MultiPolygon([vs.Polygon(_ring(10, 0, 1)), vs.Polygon(_ring(13, 0, 1, 9))]), vs.Polygon()]


def _assert_same(ga, ref):
    np.testing.assert_array_equal(ga._tags, ref._tags)
    np.testing.assert_array_equal(ga._geom_off, ref._geom_off)
    np.testing.assert_array_equal(ga._part_off, ref._part_off)
    np.testing.assert_array_equal(ga._ring_off, ref._ring_off)
    np.testing.assert_array_equal(ga._x, ref._x)
    np.testing.assert_array_equal(ga._y, ref._y)
    np.testing.assert_array_equal(ga._px, ref._px)
    np.testing.assert_array_equal(ga._py, ref._py)


def _arrow_polygons(shapes, multi=False):
    rows = []
    for s in shapes:
        if s is None:
            rows.append(None)
            continue
        polys = list(s.polygons) if isinstance(s, vs.MultiPolygon) else ([] if s.is_empty else [s])
        parts = [[[{"x": float(x), "y": float(y)} for x, y in ring] for ring in p.rings] for p in polys]
        rows.append(parts if multi else (parts[0] if parts else []))
    t = pa.list_(pa.list_(pa.list_(PT))) if multi else pa.list_(pa.list_(PT))
    return pa.array(rows, type=t)


def test_native_polygon_and_multipolygon_match_from_shapes():
    shapes = _shapes()
    poly_only = [s if not isinstance(s, vs.MultiPolygon) else None for s in shapes]
    ga = vio._native(_arrow_polygons(poly_only), "geoarrow.polygon")
    _assert_same(ga, vs.GeometryArray.from_shapes(poly_only))
    multi = [vs.MultiPolygon([s]) if isinstance(s, vs.Polygon) and not s.is_empty else s
             for s in shapes if not (isinstance(s, vs.Polygon) and s.is_empty)]
    gm = vio._native(_arrow_polygons(multi, multi=True), "geoarrow.multipolygon")
    ref = vs.GeometryArray.from_shapes(multi)
    np.testing.assert_array_equal(gm._geom_off, ref._geom_off)
    np.testing.assert_array_equal(gm._x, ref._x)
    assert (gm._tags[gm._tags >= 0] == 5).all()


def test_native_points_separated_interleaved_sliced_chunked():
    sep = pa.array([{"x": 1.0, "y": 2.0}, None, {"x": 3.0, "y": 4.0}], type=PT)
    g = vio.geometry_array_from_arrow(sep, field=pa.field("g", PT, metadata={b"ARROW:extension:name": b"geoarrow.point"}))
    assert g._tags.tolist() == [0, -1, 0] and g._px[[0, 2]].tolist() == [1.0, 3.0]
    inter = pa.array([[1.0, 2.0, 9.0], [3.0, 4.0, 9.0]], type=pa.list_(pa.float64(), 3))
    g2 = vio._native(inter, "geoarrow.point")
    assert g2._px.tolist() == [1.0, 3.0] and g2._py.tolist() == [2.0, 4.0]
    g3 = vio._native(sep.slice(2, 1), "geoarrow.point")
    assert g3._px.tolist() == [3.0]
    polys = _arrow_polygons(_shapes()[:3])
    chunked = pa.chunked_array([polys.slice(0, 2), polys.slice(2, 1)])
    g4 = vio.geometry_array_from_arrow(chunked, field=pa.field("g", polys.type, metadata={
        b"ARROW:extension:name": b"geoarrow.polygon"}))
    _assert_same(g4, vs.GeometryArray.from_shapes(_shapes()[:3]))


def test_native_geoparquet_roundtrip_with_bbox(tmp_path):
    shapes = [s for s in _shapes() if not isinstance(s, vs.MultiPolygon)]
    col = _arrow_polygons(shapes)
    meta = {"version": "1.1.0", "primary_column": "geometry",
            "columns": {"geometry": {"encoding": "polygon", "geometry_types": ["Polygon"]}}}
    table = pa.table({"name": ["a", "b", "c", "d"], "geometry": col})
    table = table.replace_schema_metadata({b"geo": json.dumps(meta).encode()})
    path = tmp_path / "p.parquet"
    pq.write_table(table, path)
    gdf = vio.read_geoparquet(path)
    assert list(gdf.columns) == ["name", "geometry"] and gdf.geometry.name == "geometry"
    _assert_same(gdf.geometry.values, vs.GeometryArray.from_shapes(shapes))
    sub = vio.read_geoparquet(path, bbox=(4, 4, 6, 6))
    assert sub["name"].tolist() == ["c"]


def test_unsupported_native_encoding_raises():
    ls = pa.array([[{"x": 0.0, "y": 0.0}]], type=pa.list_(PT))
    with pytest.raises(NotImplementedError):
        vio._native(ls, "geoarrow.linestring")


# ------------------------------------------------------------------- GPU ---

# Golden WKB vectors from the reference's own tests
GOLDEN = [
    # tests/upstream/geopandas/tests/test_array.py:157
    ("0101000000CDCCCCCCCCCC1440CDCCCCCCCC0C4A40", (5.2, 52.1)),
    # tests/test_io_arrow.py:489, :523 (big-endian)
    ("00000000013ff00000000000004000000000000000", (1.0, 2.0)),
    # tests/test_io_arrow.py:502-504 (EWKB SRID 4326)
    ("0101000020e6100000000000000000f03f0000000000000040", (1.0, 2.0)),
    # tests/test_io_arrow.py:505-507 (ISO Point Z)
    ("01e9030000000000000000f03f00000000000000400000000000000840", (1.0, 2.0)),
    # tests/test_io_arrow.py:1690-1691
    ("010100000000000000000000000000000000000000", (0.0, 0.0)),
    ("0101000000000000000000f03f000000000000f03f", (1.0, 1.0)),
]


def test_oracle_wkb_golden_points(oracle):
    data, off, valid = W.arrow_layout([bytes.fromhex(h) for h, _ in GOLDEN])
    sz, out = oracle.wkb_decode(data, off, valid)
    assert sz["n_points"] == len(GOLDEN) and sz["n_coords"] == 0
    np.testing.assert_array_equal(np.c_[out["px"], out["py"]], np.array([xy for _, xy in GOLDEN]))


def test_oracle_wkb_unsupported_and_malformed(oracle):
    gc = bytes.fromhex("010700000000000000")  # tests/test_io_arrow.py:508 (GeometryCollection)
    line = bytes.fromhex("01020000000100000000000000000008400000000000000840")  # test_array.py:167
    truncated = W.polygon([_ring(0, 0, 1)])[:-5]
    data, off, valid = W.arrow_layout([truncated, W.point(1, 2), gc, line, b"\x07", None, b""])
    sz, out = oracle.wkb_decode(data, off, valid)
    assert out["tags"].tolist() == [-1, 0, -1, -1, -1, -1, -1]
    assert (sz["n_points"], sz["n_unsupported"], sz["n_malformed"], sz["n_null"]) == (1, 2, 2, 2)
    assert sz["n_parts"] == sz["n_rings"] == sz["n_coords"] == 0


@pytest.mark.parametrize("variant", ["little", "big", "iso_z", "ewkb_zm_srid", "mixed_order_parts"])
def test_oracle_wkb_matches_from_shapes(oracle, variant):
    """The CPU decoder against the host layout built from shape objects."""
    shapes = _shapes() + [vs.Point(3.5, -1.25), None]
    kw = {"little": dict(), "big": dict(little=False), "iso_z": dict(dims="xyz"),
          "ewkb_zm_srid": dict(dims="xyzm", ewkb=True, srid=4326), "mixed_order_parts": dict(little=False)}[variant]
    vals = []
    for s in shapes:
        if s is None:
            vals.append(None)
        elif isinstance(s, vs.Point):
            vals.append(W.point(s.x, s.y, **kw))
        elif isinstance(s, vs.MultiPolygon):
            extra = {"part_little": [True, False]} if variant == "mixed_order_parts" else {}
            vals.append(W.multipolygon([p.rings for p in s.polygons], **kw, **extra))
        else:
            vals.append(W.polygon([] if s.is_empty else s.rings, **kw))
    sz, out = oracle.wkb_decode(*W.arrow_layout(vals))
    ref = vs.GeometryArray.from_shapes(shapes)
    np.testing.assert_array_equal(out["tags"], ref._tags)
    for k in ("geom_off", "part_off", "ring_off", "x", "y"):
        np.testing.assert_array_equal(out[k], getattr(ref, "_" + k))
    np.testing.assert_array_equal(out["px"][out["tags"] == 0], ref._px[ref._tags == 0])


def test_oracle_wkb_synthetic_polygons(oracle):
    """The vectorised synthetic-column writer and the CPU decoder agree."""
    from vibespatial_b200.testing import synthetic as syn

    w = syn.degenerate_join(seed=5, n_points=1_000, n_polys=400)
    sz, out = oracle.wkb_decode(*syn.wkb_polygons(w.polys))
    assert sz["n_malformed"] == sz["n_unsupported"] == 0
    for k in ("geom_off", "part_off", "ring_off", "x", "y"):
        np.testing.assert_array_equal(out[k], getattr(w.polys, k))
    data, off = syn.wkb_points(w.px, w.py)
    sz, out = oracle.wkb_decode(data, off)
    assert sz["n_points"] == w.n_points
    np.testing.assert_array_equal(out["px"], w.px)
    np.testing.assert_array_equal(out["py"], w.py)


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int64) if a.dtype == np.float64 else a


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_wkb_fuzz_matches_oracle(ctx, vsabi, oracle, seed):
    """Device decoder == CPU decoder, bit for bit, on seeded mixes of every
    encoding, nulls, other types, truncated, corrupted and junk values."""
    import torch

    rng = np.random.default_rng(seed)
    data, off, valid = W.arrow_layout(W.fuzz_values(rng, 30_000))
    sz_o, out_o = oracle.wkb_decode(data, off, valid)
    dev = torch.device("cuda", 0)
    sz_d, out_d = vsabi.wkb_decode(ctx, torch.from_numpy(data).to(dev), torch.from_numpy(off).to(dev),
                                   torch.from_numpy(valid).to(dev))
    assert sz_d == sz_o
    for k, v in out_o.items():
        np.testing.assert_array_equal(_bits(out_d[k].cpu().numpy()), _bits(v), err_msg=k)


@pytest.mark.gpu
def test_wkb_synthetic_columns_match_oracle(ctx, vsabi, oracle):
    """Large single-encoding columns (the ingest benchmark's layout)."""
    import torch

    from vibespatial_b200.testing import synthetic as syn

    w = syn.zipf_join(seed=3, n_points=2_000_000, n_polys=100_000)
    dev = torch.device("cuda", 0)
    for data, off in (syn.wkb_polygons(w.polys), syn.wkb_points(w.px, w.py)):
        sz_o, out_o = oracle.wkb_decode(data, off)
        sz_d, out_d = vsabi.wkb_decode(ctx, torch.from_numpy(data).to(dev), torch.from_numpy(off).to(dev))
        assert sz_d == sz_o
        for k, v in out_o.items():
            np.testing.assert_array_equal(_bits(out_d[k].cpu().numpy()), _bits(v), err_msg=k)


@pytest.mark.gpu
def test_wkb_golden_points():
    ga = vio.from_wkb([bytes.fromhex(h) for h, _ in GOLDEN])
    assert (ga._tags == 0).all()
    np.testing.assert_array_equal(np.c_[ga._px, ga._py], np.array([xy for _, xy in GOLDEN]))


@pytest.mark.gpu
def test_wkb_unsupported_and_malformed():
    gc = bytes.fromhex("010700000000000000")  # tests/test_io_arrow.py:508 (GeometryCollection)
    line = bytes.fromhex("01020000000100000000000000000008400000000000000840")  # test_array.py:167
    with pytest.raises(NotImplementedError):
        vio.from_wkb([gc])
    with pytest.raises(NotImplementedError):
        vio.from_wkb([line])
    truncated = W.polygon([_ring(0, 0, 1)])[:-5]
    with pytest.raises(ValueError):
        vio.from_wkb([truncated])
    ga = vio.from_wkb([truncated, W.point(1, 2), gc, b"\x07", None], on_invalid="ignore")
    assert ga._tags.tolist() == [-1, 0, -1, -1, -1]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["little", "big", "iso_z", "ewkb_zm_srid", "mixed_order_parts"])
def test_wkb_roundtrip_matches_from_shapes(variant):
    shapes = _shapes() + [vs.Point(3.5, -1.25), None, vs.Point(np.nan, np.nan)]
    kw = {"little": dict(), "big": dict(little=False), "iso_z": dict(dims="xyz"),
          "ewkb_zm_srid": dict(dims="xyzm", ewkb=True, srid=4326), "mixed_order_parts": dict(little=False)}[variant]
    vals = []
    for s in shapes:
        if s is None:
            vals.append(None)
        elif isinstance(s, vs.Point):
            vals.append(W.point(s.x, s.y, **kw))
        elif isinstance(s, vs.MultiPolygon):
            parts = [p.rings for p in s.polygons]
            extra = {"part_little": [True, False]} if variant == "mixed_order_parts" else {}
            vals.append(W.multipolygon(parts, **kw, **extra))
        else:
            vals.append(W.polygon([] if s.is_empty else s.rings, **kw))
    ga = vio.from_wkb(vals)
    ref = vs.GeometryArray.from_shapes(shapes)
    np.testing.assert_array_equal(ga._tags, ref._tags)
    np.testing.assert_array_equal(ga._geom_off, ref._geom_off)
    np.testing.assert_array_equal(ga._part_off, ref._part_off)
    np.testing.assert_array_equal(ga._ring_off, ref._ring_off)
    np.testing.assert_array_equal(ga._x, ref._x)
    np.testing.assert_array_equal(ga._y, ref._y)
    np.testing.assert_array_equal(ga._px[ga._tags == 0], ref._px[ref._tags == 0])
    # through an Arrow binary array (sliced) as well
    arr = pa.array([None] + vals, type=pa.binary()).slice(1)
    _assert_same(vio.from_wkb(arr), ga)


@pytest.mark.gpu
def test_wkb_geoparquet_join_matches_oracle(tmp_path, oracle):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=4, n_points=20_000, n_polys=300)
    polys = []
    for g in range(len(w.polys.geom_off) - 1):
        r0 = w.polys.part_off[w.polys.geom_off[g]]
        r1 = w.polys.part_off[w.polys.geom_off[g + 1]]
        rings = [np.c_[w.polys.x[w.polys.ring_off[r]:w.polys.ring_off[r + 1]],
                       w.polys.y[w.polys.ring_off[r]:w.polys.ring_off[r + 1]]] for r in range(r0, r1)]
        polys.append(W.polygon(rings, little=bool(g % 2)))
    pts = [W.point(x, y) for x, y in zip(w.px, w.py)]
    meta = {"version": "1.1.0", "primary_column": "geometry",
            "columns": {"geometry": {"encoding": "WKB", "geometry_types": []}}}
    for name, vals in (("polys", polys), ("pts", pts)):
        t = pa.table({"row": np.arange(len(vals)), "geometry": pa.array(vals, type=pa.binary())})
        pq.write_table(t.replace_schema_metadata({b"geo": json.dumps(meta).encode()}), tmp_path / f"{name}.parquet")
    gp = vio.read_geoparquet(tmp_path / "polys.parquet")
    gpts = vio.read_geoparquet(tmp_path / "pts.parquet")
    out = vs.sjoin(gpts, gp, predicate="within")
    el, er = oracle.join(w.px, w.py, None, oracle.Polygons(w.polys.x, w.polys.y, w.polys.ring_off,
                                                           w.polys.part_off, w.polys.geom_off), "within")
    got = np.lexsort((out["index_right"].to_numpy(), out.index.to_numpy()))
    np.testing.assert_array_equal(out.index.to_numpy()[got], el)
    np.testing.assert_array_equal(out["index_right"].to_numpy()[got], er)
