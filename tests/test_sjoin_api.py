"""The GeoPandas-compatible surface: sjoin, GeoSeries.within/contains, sindex.query.

Each test runs twice: with the CPU oracle as the pair / location source
(checks the host logic: predicate routing, frame assembly, index naming,
suffixes, how='left'/'right'/'outer', on_attribute) and on the GPU through
the C-ABI (marked gpu).  Expected shapes and values come from the reference's
vendored GeoPandas test-suite (tests/upstream/geopandas/tools/tests/test_sjoin.py).
"""
import json
from pathlib import Path

import numpy as np
import pandas as pd
import pytest

import vibespatial_b200 as vs
from vibespatial_b200 import predicates as vs_predicates
from vibespatial_b200 import query as vs_query
from vibespatial_b200.geometry import GeometryArray

GOLDEN = Path(__file__).resolve().parent / "golden"
EXP = json.loads((GOLDEN / "expected.json").read_text())


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request, monkeypatch, oracle):
    if request.param == "oracle":
        def pairs(points, polygons, predicate):
            px, py, pv = points.point_buffers()
            pb = polygons.polygon_buffers()
            P = oracle.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)
            left, right = oracle.join(px, py, pv, P, predicate)
            return left.astype(np.intp), right.astype(np.intp)

        def locate(points, polygons):
            px, py, pv = points.point_buffers()
            pb = polygons.polygon_buffers()
            P = oracle.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)
            return oracle.locate_aligned(px, py, pv, P)

        def dwithin(points, polygons, distance=0.0, point_distance=None, geom_distance=None):
            px, py, pv = points.point_buffers()
            pb = polygons.polygon_buffers()
            P = oracle.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)
            left, right, _ = oracle.dwithin_join(px, py, pv, P, distance, point_distance=point_distance,
                                                 geom_distance=geom_distance)
            return left.astype(np.intp), right.astype(np.intp)

        def nearest(points, polygons, max_distance=None):
            px, py, pv = points.point_buffers()
            pb = polygons.polygon_buffers()
            P = oracle.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)
            md = float("inf") if max_distance is None else max_distance
            left, right, dist = oracle.nearest_join(px, py, pv, P, md)
            return left.astype(np.intp), right.astype(np.intp), dist

        monkeypatch.setattr(vs_query, "_pairs_backend", pairs)
        monkeypatch.setattr(vs_query, "_dwithin_backend", dwithin)
        def nearest_polygons(polygons, points, max_distance=None):
            px, py, pv = points.point_buffers()
            pb = polygons.polygon_buffers()
            P = oracle.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)
            md = float("inf") if max_distance is None else max_distance
            left, right, dist = oracle.nearest_polygons_join(px, py, pv, P, md)
            return left.astype(np.intp), right.astype(np.intp), dist

        monkeypatch.setattr(vs_query, "_nearest_backend", nearest)
        monkeypatch.setattr(vs_query, "_nearest_polygons_backend", nearest_polygons)
        def distances(points, polygons):
            px, py, pv = points.point_buffers()
            pb = polygons.polygon_buffers()
            P = oracle.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)
            return oracle.distance_aligned(px, py, pv, P)

        monkeypatch.setattr(vs_predicates, "_locate_backend", locate)
        monkeypatch.setattr(vs_predicates, "_distance_backend", distances)
    return request.param


def nybb_frames():
    d = dict(np.load(GOLDEN / "nybb.npz"))
    geoms = GeometryArray.from_polygon_buffers(d["x"], d["y"], d["ring_off"], d["part_off"], d["geom_off"],
                                               geom_type=d["geom_type"])
    polydf = vs.GeoDataFrame({"BoroCode": d["attr_BoroCode"], "BoroName": d["attr_BoroName"],
                              "Shape_Leng": d["attr_Shape_Leng"], "Shape_Area": d["attr_Shape_Area"]},
                             geometry=geoms, crs="EPSG:2263")
    b = [int(v) for v in polydf.total_bounds]
    n = 20
    xs = list(range(b[0], b[2], int((b[2] - b[0]) / n)))
    ys = list(range(b[1], b[3], int((b[3] - b[1]) / n)))
    pts = list(zip(xs, ys))
    pointdf = vs.GeoDataFrame({"geometry": [vs.Point(x, y) for x, y in pts],
                               "pointattr1": [x + y for x, y in pts], "pointattr2": [x - y for x, y in pts]},
                              crs="EPSG:2263")
    return pointdf, polydf


def test_nybb_left_within(backend):
    pointdf, polydf = nybb_frames()
    df = vs.sjoin(pointdf, polydf, how="left", predicate="within")
    assert list(df.shape) == EXP["nybb_within_left_shape"]["value"]
    assert df.loc[1]["BoroName"] == EXP["nybb_within_left_row1_boro"]["value"]
    assert set(df.geometry.geom_type) == {"Point"}
    assert "pointattr1" in df.columns and "BoroCode" in df.columns and "index_right" in df.columns
    # points contain polygons? never: all right columns missing
    df2 = vs.sjoin(pointdf, polydf, how="left", predicate="contains")
    assert df2.shape == (21, 8) and np.isnan(df2.loc[1]["Shape_Area"])


def test_nybb_inner_and_right(backend):
    pointdf, polydf = nybb_frames()
    assert list(vs.sjoin(pointdf, polydf, how="inner").shape) == EXP["nybb_inner_intersects_shape"]["value"]
    df = vs.sjoin(pointdf, polydf, how="right")
    df2 = vs.sjoin(polydf, pointdf, how="left")
    assert list(df.shape) == EXP["nybb_right_intersects_shape"]["value"]
    assert df.shape == df2.shape
    assert set(df.geometry.geom_type) == {"MultiPolygon"}
    assert set(df2.geometry.geom_type) == {"MultiPolygon"}
    assert list(df.columns[:1]) == ["index_left"]


def test_nybb_geometry_name_and_duplicate_columns(backend):
    pointdf, polydf = nybb_frames()
    renamed = polydf.rename_geometry("new_geom")
    res = vs.sjoin(renamed, pointdf, how="left")
    assert res.geometry.name == "new_geom"
    pointdf2 = pointdf.rename(columns={"pointattr1": "Shape_Area"})
    df = vs.sjoin(pointdf2, polydf, how="left")
    assert "Shape_Area_left" in df.columns and "Shape_Area_right" in df.columns
    with pytest.raises(ValueError):
        vs.sjoin(pointdf, polydf, how="left", predicate="spandex")
    with pytest.raises(ValueError, match="`how` was"):
        vs.sjoin(pointdf, polydf, how="abcde")
    with pytest.raises(TypeError):
        vs.sjoin(pointdf, polydf, unknown=1)


@pytest.mark.parametrize("how", ["left", "right", "inner"])
def test_nybb_named_index(backend, how):
    """Index names pass through untouched (tests/upstream/geopandas/tools/tests/test_sjoin.py:911-927)."""
    pointdf, polydf = nybb_frames()
    pointdf.index.name = "pointid"
    polydf.index.name = "polyid"
    res = vs.sjoin(pointdf, polydf, how=how)
    assert pointdf.index.name == "pointid" and polydf.index.name == "polyid"
    assert res.index.name == ("polyid" if how == "right" else "pointid")


def test_nybb_values_outer_and_empty_geometries(backend):
    """test_sjoin.py:929-1008: a non-default polygon index, the outer join's
    counts, and empty geometries (of another family) that never match."""
    pointdf, polydf = nybb_frames()
    relabelled = polydf.copy()
    relabelled.index = [1, 3, 4, 5, 6]
    assert vs.sjoin(pointdf, relabelled, how="left").shape == (21, 8)
    assert vs.sjoin(relabelled, pointdf, how="left").shape == (12, 8)

    df = vs.sjoin(pointdf, polydf, how="outer")
    left = vs.sjoin(pointdf, polydf, how="left")
    right = vs.sjoin(pointdf, polydf, how="right")
    unmatched_left = int(left["index_right"].isna().sum())
    unmatched_right = int(right["index_left"].isna().sum())
    assert len(df) == len(left) + unmatched_right
    assert int(df["index_left"].isna().sum()) == unmatched_right
    assert int(df["index_right"].isna().sum()) == unmatched_left
    assert df.geometry.notna().all()

    # the reference uses empty GeometryCollections; empty polygons play that part here
    empty = vs.GeoDataFrame(geometry=GeometryArray.from_shapes([vs.Polygon([])] * 3), crs=pointdf.crs)
    assert vs.sjoin(pd.concat([pointdf, empty]), polydf, how="left").shape == (24, 8)
    assert vs.sjoin(pointdf, pd.concat([polydf, empty]), how="left").shape == (21, 8)


@pytest.mark.parametrize("how, lsuffix, rsuffix, expected_cols", [
    ("left", "left", "right", {"col_left", "col_right", "index_right"}),
    ("inner", "left", "right", {"col_left", "col_right", "index_right"}),
    ("right", "left", "right", {"col_left", "col_right", "index_left"}),
    ("outer", "left", "right", {"col_left", "col_right", "index_left", "index_right"}),
    ("left", "lft", "rgt", {"col_lft", "col_rgt", "index_rgt"}),
    ("inner", "lft", "rgt", {"col_lft", "col_rgt", "index_rgt"}),
    ("right", "lft", "rgt", {"col_lft", "col_rgt", "index_lft"}),
    ("outer", "lft", "rgt", {"col_lft", "col_rgt", "index_lft", "index_rgt"}),
])
def test_suffixes(backend, how, lsuffix, rsuffix, expected_cols):
    """tests/upstream/geopandas/tools/tests/test_sjoin.py:141-163, with a point
    and a polygon around it (the reference uses two points)."""
    left = vs.GeoDataFrame({"col": [1], "geometry": [vs.Point(0, 0)]})
    right = vs.GeoDataFrame({"col": [1], "geometry": [vs.box(-1, -1, 1, 1)]})
    joined = vs.sjoin(left, right, how=how, lsuffix=lsuffix, rsuffix=rsuffix)
    assert set(joined.columns) == expected_cols | {"geometry"}


def test_suffix_creating_duplicate_columns_warns(backend):
    """A suffix that renames an overlapping column onto another column of the same frame warns
    (GeoPandas' deprecation, src/vibespatial/api/_native_results.py:355-375); plain overlaps do not."""
    import warnings

    left = vs.GeoDataFrame({"col": [1], "col_left": [2], "geometry": [vs.Point(0, 0)]})
    right = vs.GeoDataFrame({"col": [3], "geometry": [vs.box(-1, -1, 1, 1)]})
    with pytest.warns(FutureWarning, match="Passing 'suffixes' which cause duplicate columns {'col_left'}"):
        joined = vs.sjoin(left, right)
    assert list(joined.columns).count("col_left") == 2
    left = vs.GeoDataFrame({"col": [1], "other": [2], "geometry": [vs.Point(0, 0)]})
    with warnings.catch_warnings():
        warnings.simplefilter("error", FutureWarning)
        vs.sjoin(left, right)


def test_argument_errors_and_crs_warning(backend):
    """test_sjoin.py:165-181, 325-344: a CRS mismatch warns, unknown keywords
    and non-frame inputs raise."""
    left = vs.GeoDataFrame({"col": [1], "geometry": [vs.Point(0, 0)]}, crs="EPSG:3857")
    right = vs.GeoDataFrame({"col": [1], "geometry": [vs.box(-1, -1, 1, 1)]}, crs="EPSG:4326")
    with pytest.warns(UserWarning, match="CRS mismatch between the CRS"):
        vs.sjoin(left, right)
    right = vs.GeoDataFrame({"col": [1], "geometry": [vs.box(-1, -1, 1, 1)]}, crs="EPSG:3857")
    with pytest.raises(TypeError, match=r"sjoin\(\) got an unexpected keyword argument 'extra_param'"):
        vs.sjoin(left, right, extra_param="test")
    with pytest.raises(ValueError, match="'left_df' should be GeoDataFrame"):
        vs.sjoin(left.geometry, right)
    with pytest.raises(ValueError, match="'right_df' should be GeoDataFrame"):
        vs.sjoin(left, right.geometry)


PREDICATES_ALL = ["contains", "contains_properly", "covered_by", "covers", "crosses", "intersects", "touches",
                  "within"]


@pytest.mark.parametrize("predicate", PREDICATES_ALL)
@pytest.mark.parametrize("empty_kind", ["empty geometries", "no rows"])
def test_join_with_empty(backend, predicate, empty_kind):
    """test_sjoin.py:267-323: a point outside both polygons, a frame of empty
    geometries and a frame without rows give all-missing or empty joins."""
    polygons = vs.GeoDataFrame({"col2": [1, 2], "geometry": [vs.box(0, 0, 1, 1), vs.box(1, 0, 2, 1)]})
    not_in = vs.GeoDataFrame({"col1": [1], "geometry": [vs.Point(-0.5, 0.5)]})
    assert vs.sjoin(not_in, polygons, how="left", predicate=predicate).index_right.isnull().all()
    assert vs.sjoin(not_in, polygons, how="right", predicate=predicate).index_left.isnull().all()
    assert vs.sjoin(not_in, polygons, how="inner", predicate=predicate).empty
    if empty_kind == "empty geometries":
        empty = vs.GeoDataFrame(geometry=GeometryArray.from_shapes([vs.Point(), vs.Point()]))
    else:
        empty = vs.GeoDataFrame(geometry=GeometryArray.from_shapes([]))
    result = vs.sjoin(empty, polygons, how="left", predicate=predicate)
    assert result.index_right.isnull().all()
    result = vs.sjoin(empty, polygons, how="right", predicate=predicate)
    assert result.index_left.isnull().all()
    assert vs.sjoin(empty, polygons, how="inner", predicate=predicate).empty


@pytest.mark.parametrize("how", ["inner", "left", "right"])
def test_preserve_index_names(backend, how):
    """test_sjoin.py:610-645 with boxes around the right-hand points: both
    index names survive, and equal names get the suffixes."""
    pts = [vs.Point(1, 1), vs.Point(2, 2)]
    boxes = [vs.box(0.5, 0.5, 1.5, 1.5), vs.box(1.5, 1.6, 2.5, 2.5)]
    df1 = vs.GeoDataFrame({"geometry": pts}, index=pd.Index([1, 2], name="myidx1"))
    df2 = vs.GeoDataFrame({"geometry": boxes}, index=pd.Index(["a", "b"], name="myidx2"))
    result = vs.sjoin(df1, df2, how=how)
    if how in ("inner", "left"):
        assert result.index.name == "myidx1" and result.index.tolist() == [1, 2]
        assert list(result.columns) == ["geometry", "myidx2"] and result["myidx2"].tolist() == ["a", "b"]
    else:
        assert result.index.name == "myidx2" and result.index.tolist() == ["a", "b"]
        assert list(result.columns) == ["myidx1", "geometry"] and result["myidx1"].tolist() == [1, 2]
    df1.index.name = "myidx"
    df2.index.name = "myidx"
    result = vs.sjoin(df1, df2, how=how)
    if how in ("inner", "left"):
        assert result.index.name == "myidx_left" and list(result.columns) == ["geometry", "myidx_right"]
    else:
        assert result.index.name == "myidx_right" and list(result.columns) == ["myidx_left", "geometry"]


@pytest.mark.parametrize("how", ["inner", "left", "right"])
def test_duplicate_column_index_name(backend, how):
    """test_sjoin.py:705-739: a left column named like the right index gets
    the suffixes on both."""
    pts = [vs.Point(1, 1), vs.Point(2, 2)]
    boxes = [vs.box(0.5, 0.5, 1.5, 1.5), vs.box(1.5, 1.6, 2.5, 2.5)]
    df1 = vs.GeoDataFrame({"myidx": [1, 2], "geometry": pts})
    df2 = vs.GeoDataFrame({"geometry": boxes}, index=pd.Index(["a", "b"], name="myidx"))
    result = vs.sjoin(df1, df2, how=how)
    if how in ("inner", "left"):
        assert list(result.columns) == ["myidx_left", "geometry", "myidx_right"]
        assert result["myidx_left"].tolist() == [1, 2] and result["myidx_right"].tolist() == ["a", "b"]
    else:
        assert result.index.name == "myidx_right" and result.index.tolist() == ["a", "b"]
        assert list(result.columns) == ["index_left", "myidx_left", "geometry"]
    result = vs.sjoin(df2, df1, how=how)
    if how in ("inner", "left"):
        assert result.index.name == "myidx_left" and result.index.tolist() == ["a", "b"]
        assert list(result.columns) == ["geometry", "index_right", "myidx_right"]
        assert result["myidx_right"].tolist() == [1, 2]
    else:
        assert list(result.columns) == ["myidx_left", "myidx_right", "geometry"]
        assert result["myidx_left"].tolist() == ["a", "b"] and result["myidx_right"].tolist() == [1, 2]


@pytest.mark.parametrize("how", ["inner", "left", "right"])
def test_conflicting_column_names(backend, how):
    """test_sjoin.py:792-835: a column named like the generated index column
    raises; a column named like a suffixed one is kept beside it."""
    pts = [vs.Point(1, 1), vs.Point(2, 2)]
    boxes = [vs.box(0.5, 0.5, 1.5, 1.5), vs.box(1.5, 1.6, 2.5, 2.5)]
    df1 = vs.GeoDataFrame({"index_right": [1, 2], "geometry": pts})
    df2 = vs.GeoDataFrame({"geometry": boxes})
    with pytest.raises(ValueError, match="'index_right' cannot be a column name"):
        vs.sjoin(df1, df2, how=how)
    df1 = vs.GeoDataFrame({"column": [1, 2], "column_right": ["a", "b"], "geometry": pts})
    df2 = vs.GeoDataFrame({"column": [0.1, 0.2], "geometry": boxes})
    result = vs.sjoin(df1, df2, how=how)
    if how in ("inner", "left"):
        assert list(result.columns) == ["column_left", "column_right", "geometry", "index_right", "column_right"]
    else:
        assert list(result.columns) == ["index_left", "column_left", "column_right", "column_right", "geometry"]


def test_no_valid_geoms(backend):
    pointdf, polydf = nybb_frames()
    empty = vs.GeoDataFrame(geometry=GeometryArray.from_shapes([]), crs=pointdf.crs)
    for predicate in ("intersects", "within", "contains"):
        assert vs.sjoin(pointdf, empty, how="inner", predicate=predicate).empty
        assert vs.sjoin(pointdf, empty, how="right", predicate=predicate).empty
        assert vs.sjoin(empty, pointdf, how="inner", predicate=predicate).empty
        assert vs.sjoin(empty, pointdf, how="left", predicate=predicate).empty


def test_cities_countries(backend):
    w = dict(np.load(GOLDEN / "naturalearth_lowres.npz"))
    c = dict(np.load(GOLDEN / "naturalearth_cities.npz"))
    world = vs.GeoDataFrame({"name": w["attr_name"]},
                            geometry=GeometryArray.from_polygon_buffers(w["x"], w["y"], w["ring_off"], w["part_off"],
                                                                        w["geom_off"], geom_type=w["geom_type"]))
    cities = vs.GeoDataFrame({"name": c["attr_name"]}, geometry=vs.points_from_xy(c["x"], c["y"]))
    countries = world[["geometry", "name"]].rename(columns={"name": "country"})
    out = vs.sjoin(cities, countries, how="inner", predicate="intersects")
    assert list(out.shape) == EXP["cities_countries_inner_intersects_shape"]["value"]
    # within == contains with the sides swapped
    a = vs.sjoin(cities, countries, predicate="within")
    b = vs.sjoin(countries, cities, predicate="contains")
    assert sorted(zip(a.index, a["index_right"])) == sorted(zip(b["index_right"], b.index))


def test_cities_countries_shared_attribute(backend):
    """on_attribute: cities and countries joined where they intersect and
    their names share a first letter (the reference's known answer: 23 rows,
    5 columns), through the device export when the pairs are on the device."""
    w = dict(np.load(GOLDEN / "naturalearth_lowres.npz"))
    c = dict(np.load(GOLDEN / "naturalearth_cities.npz"))
    countries = vs.GeoDataFrame({"country": w["attr_name"]},
                                geometry=GeometryArray.from_polygon_buffers(w["x"], w["y"], w["ring_off"],
                                                                            w["part_off"], w["geom_off"],
                                                                            geom_type=w["geom_type"]))
    cities = vs.GeoDataFrame({"name": c["attr_name"]}, geometry=vs.points_from_xy(c["x"], c["y"]))
    countries["firstLetter"] = countries["country"].astype(str).str[0]
    cities["firstLetter"] = cities["name"].astype(str).str[0]
    result = vs.sjoin(cities, countries, on_attribute="firstLetter")
    assert (result["country"].astype(str).str[0] == result["name"].astype(str).str[0]).all()
    assert list(result.shape) == EXP["cities_countries_shared_first_letter_shape"]["value"]


@pytest.mark.parametrize("predicate", ["contains", "contains_properly", "covered_by", "covers", "crosses",
                                       "intersects", "touches", "within"])
def test_sjoin_left_order(backend, predicate):
    """A left join keeps the points' order, whatever the predicate
    (tests/upstream/geopandas/tools/tests/test_sjoin.py:480-511)."""
    pts = vs.GeoDataFrame(geometry=vs.points_from_xy([0.1, 0.4, 0.3, 0.7], [0.8, 0.6, 0.9, 0.1]))
    polys = vs.GeoDataFrame({"id": [1, 2, 3, 4]},
                            geometry=[vs.box(0, 0, 0.5, 0.5), vs.box(0, 0.5, 0.5, 1), vs.box(0.5, 0, 1, 0.5),
                                      vs.box(0.5, 0.5, 1, 1)])
    joined = vs.sjoin(pts, polys, predicate=predicate, how="left")
    pd.testing.assert_index_equal(joined.index, pts.index)
    if predicate in ("intersects", "within", "covered_by"):
        # each point lies inside exactly one box
        assert joined["id"].tolist() == [2, 2, 2, 3]


def _small_frames(index_kind):
    polys = vs.GeoDataFrame({"geometry": [vs.box(0, 0, 5, 5), vs.box(3, 3, 6, 6), vs.box(10, 10, 11, 11)],
                             "df2": [3, 4, 5]})
    pts = vs.GeoDataFrame({"geometry": [vs.Point(1, 1), vs.Point(4, 4), vs.Point(20, 20), vs.Point(5, 5)],
                           "df1": [0, 1, 2, 3]})
    if index_kind == "string-index":
        pts.index = ["a", "b", "c", "d"]
        polys.index = ["e", "f", "g"]
    elif index_kind == "named-index":
        pts.index.name = "df1_ix"
        polys.index.name = "df2_ix"
    elif index_kind == "multi-index":
        pts = pts.set_index([["a", "b", "c", "d"], ["p", "q", "r", "s"]])
        polys = polys.set_index([["e", "f", "g"], ["x", "y", "z"]])
    return pts, polys


@pytest.mark.parametrize("index_kind", ["default-index", "string-index", "named-index", "multi-index"])
def test_index_naming_and_pairs(backend, index_kind):
    pts, polys = _small_frames(index_kind)
    res = vs.sjoin(pts, polys, how="inner", predicate="intersects")
    # (1,1) in box0; (4,4) in box0 and box1; (5,5) on the boundary of box0, inside box1
    assert res["df1"].tolist() == [0, 1, 1, 3, 3]
    assert res["df2"].tolist() == [3, 3, 4, 3, 4]
    within = vs.sjoin(pts, polys, how="inner", predicate="within")
    assert within["df1"].tolist() == [0, 1, 1, 3]  # (5,5) is on box0's boundary: not within
    if index_kind == "default-index":
        assert "index_right" in res.columns and list(res.index) == [0, 1, 1, 3, 3]
    elif index_kind == "named-index":
        assert res.index.name == "df1_ix" and "df2_ix" in res.columns
    elif index_kind == "multi-index":
        assert res.index.nlevels == 2 and "index_right0" in res.columns and "index_right1" in res.columns
    left = vs.sjoin(pts, polys, how="left", predicate="within")
    assert len(left) == 5 and left["df2"].isna().sum() == 1
    right = vs.sjoin(pts, polys, how="right", predicate="within")
    assert len(right) == 5 and right["df1"].isna().sum() == 1  # box2 has no point
    outer = vs.sjoin(pts, polys, how="outer", predicate="within")
    assert len(outer) == 6  # 4 matches + point (20,20) alone + box2 alone
    assert outer.geometry.isna().sum() == 0


def test_on_attribute(backend):
    pts = vs.GeoDataFrame({"geometry": [vs.Point(1, 1), vs.Point(4, 4)], "city": ["a", "b"]})
    polys = vs.GeoDataFrame({"geometry": [vs.box(0, 0, 5, 5), vs.box(0, 0, 5, 5)], "city": ["a", "b"]})
    res = vs.sjoin(pts, polys, predicate="within", on_attribute="city")
    assert list(zip(res.index, res["index_right"])) == [(0, 0), (1, 1)]
    with pytest.raises(ValueError, match="missing"):
        vs.sjoin(pts, polys, on_attribute="nope")


def test_elementwise_within_contains(backend):
    polys = vs.GeoSeries([vs.box(0, 0, 2, 2), vs.Polygon(), None, vs.box(5, 1, 9, 3),
                          vs.Polygon([(0, 0), (4, 0), (4, 4), (0, 4)])])
    pts = vs.GeoSeries([None, vs.Point(), vs.Point(1, 1), vs.Point(8, 2), vs.Point(4, 2)])
    # nulls / empties are False; (4, 2) is on the boundary: covered_by but not within
    assert pts.within(polys).tolist() == [False, False, False, True, False]
    assert pts.covered_by(polys).tolist() == [False, False, False, True, True]
    assert polys.contains(pts).tolist() == [False, False, False, True, False]
    assert polys.covers(pts).tolist() == [False, False, False, True, True]
    assert pts.touches(polys).tolist() == [False, False, False, False, True]
    assert polys.contains_properly(pts).tolist() == [False, False, False, True, False]
    assert not pts.crosses(polys).any() and not polys.overlaps(pts).any()
    # disjoint: the empty pair is disjoint, missing rows are not, the boundary point intersects
    assert pts.disjoint(polys).tolist() == [False, True, False, False, False]
    assert polys.disjoint(vs.GeoSeries([vs.Point(3, 3)] * 5)).tolist() == [True, True, False, True, False]
    # scalar broadcast and index alignment
    s = vs.GeoSeries([vs.Point(1, 1), vs.Point(3, 3)], index=[10, 20])
    assert s.within(vs.box(0, 0, 2, 2)).tolist() == [True, False]
    p = vs.GeoSeries([vs.box(0, 0, 2, 2)], index=[20])
    aligned = s.within(p)
    assert aligned.index.tolist() == [10, 20] and aligned.tolist() == [False, False]


def test_sindex_query(backend):
    tree = vs.GeometryArray.from_shapes([vs.box(0, 0, 5, 5), vs.box(3, 3, 6, 6), vs.box(10, 10, 11, 11)])
    q = vs.GeometryArray.from_shapes([vs.Point(1, 1), vs.Point(4, 4), vs.Point(20, 20)])
    res = tree.sindex.query(q, predicate="intersects")
    # tests/test_spatial_query.py:2787-2848
    assert res[0].tolist() == [0, 1, 1] and res[1].tolist() == [0, 0, 1]
    # points as the tree, polygons as the input: contains
    res2 = q.sindex.query(tree, predicate="contains")
    assert res2[0].tolist() == [0, 0, 1] and res2[1].tolist() == [0, 1, 1]
    assert tree.sindex.query(q, predicate="contains").shape == (2, 0)
    with pytest.raises(NotImplementedError):
        tree.sindex.query(tree, predicate="intersects")


def test_sindex_query_output_formats(backend):
    tree = vs.GeometryArray.from_shapes([vs.box(0, 0, 5, 5), vs.box(3, 3, 6, 6), vs.box(10, 10, 11, 11)])
    q = vs.GeometryArray.from_shapes([vs.Point(1, 1), vs.Point(4, 4), vs.Point(20, 20)])
    dense = tree.sindex.query(q, predicate="intersects", output_format="dense")
    assert dense.shape == (3, 3) and dense.dtype == bool
    assert np.argwhere(dense).tolist() == [[0, 0], [0, 1], [1, 1]]  # (tree row, input row)
    sparse = tree.sindex.query(q, predicate="intersects", output_format="sparse")
    assert sparse.shape == (3, 3) and sparse.nnz == 3
    np.testing.assert_array_equal(sparse.toarray(), dense)
    # a scalar input: tree rows, a (len(tree),) mask, a 1-D sparse array
    assert tree.sindex.query(vs.Point(4, 4), predicate="within").tolist() == [0, 1]
    d1 = tree.sindex.query(vs.Point(4, 4), predicate="within", output_format="dense")
    assert d1.tolist() == [True, True, False]
    s1 = tree.sindex.query(vs.Point(4, 4), predicate="within", output_format="sparse")
    assert s1.shape == (3,) and s1.nnz == 2
    with pytest.raises(ValueError):
        tree.sindex.query(q, output_format="bogus")
    with pytest.raises(ValueError):
        tree.sindex.query(q, output_format="dense", return_device=True)


@pytest.mark.gpu
def test_sindex_query_return_device(backend):
    if backend != "gpu":
        pytest.skip("device output needs the CUDA join")
    tree = vs.GeometryArray.from_shapes([vs.box(0, 0, 5, 5), vs.box(3, 3, 6, 6), vs.box(10, 10, 11, 11)])
    q = vs.GeometryArray.from_shapes([vs.Point(1, 1), vs.Point(4, 4), vs.Point(20, 20)])
    rows, trees = tree.sindex.query(q, predicate="intersects", return_device=True)
    assert rows.is_cuda and trees.is_cuda
    assert rows.cpu().tolist() == [0, 1, 1] and trees.cpu().tolist() == [0, 0, 1]
    # points as the tree: pairs swapped and re-sorted on the device
    r2, t2 = q.sindex.query(tree, predicate="contains", return_device=True)
    assert r2.cpu().tolist() == [0, 0, 1] and t2.cpu().tolist() == [0, 1, 1]


# ------------------------------------------------------------ distance joins

def _distance_frames():
    # unit squares; the second has a hole; points inside, on edges, in the hole and outside
    polys = vs.GeoDataFrame({"geometry": [vs.box(0, 0, 1, 1),
                                          vs.Polygon([(3, 0), (6, 0), (6, 3), (3, 3), (3, 0)],
                                                     [[(4, 1), (4, 2), (5, 2), (5, 1), (4, 1)]]),
                                          vs.box(10, 10, 11, 11)],
                             "pid": [10, 11, 12]})
    pts = vs.GeoDataFrame({"geometry": [vs.Point(0.5, 0.5), vs.Point(2, 0.5), vs.Point(4.5, 1.5), vs.Point(1, 1),
                                        vs.Point(-3, -4), vs.Point(8, 8)],
                           "qid": [0, 1, 2, 3, 4, 5]})
    return pts, polys


def test_sjoin_dwithin(backend):
    pts, polys = _distance_frames()
    res = vs.sjoin(pts, polys, predicate="dwithin", distance=1.0)
    # (0.5,0.5) inside square 0; (2,0.5) is 1 from square 0 and 1 from polygon 1; (4.5,1.5) sits in the hole,
    # 0.5 from the hole's edges; (1,1) on square 0's corner; (-3,-4) is 5 away; (8,8) is sqrt(8) from box 2
    assert sorted(zip(res.index, res["index_right"])) == [(0, 0), (1, 0), (1, 1), (2, 1), (3, 0)]
    res = vs.sjoin(pts, polys, predicate="dwithin", distance=5.0)
    assert (4, 0) in set(zip(res.index, res["index_right"]))
    # per-row distances (one per left row)
    d = np.array([0.0, 0.5, 0.5, 0.0, 4.999999, 2.9])
    res = vs.sjoin(pts, polys, predicate="dwithin", distance=d)
    assert sorted(zip(res.index, res["index_right"])) == [(0, 0), (2, 1), (3, 0), (5, 2)]
    # polygons on the left: one distance per polygon row
    res = vs.sjoin(polys, pts, predicate="dwithin", distance=np.array([0.0, 0.5, 3.0]))
    assert sorted(zip(res.index, res["index_right"])) == [(0, 0), (0, 3), (1, 2), (2, 5)]
    with pytest.raises(ValueError):
        vs.sjoin(pts, polys, predicate="dwithin")
    with pytest.raises(ValueError):
        vs.sjoin(pts, polys, predicate="dwithin", distance=np.ones(3))
    with pytest.raises(ValueError):
        vs.sjoin(pts, polys, predicate="intersects", distance=1.0)
    # negative / NaN distances match nothing
    assert vs.sjoin(pts, polys, predicate="dwithin", distance=-1.0).empty
    assert vs.sjoin(pts, polys, predicate="dwithin", distance=np.full(6, np.nan)).empty
    # sindex.query with dwithin
    tree = polys.geometry.array
    q = pts.geometry.array
    r = tree.sindex.query(q, predicate="dwithin", distance=1.0)
    assert r[0].tolist() == [0, 1, 1, 2, 3] and r[1].tolist() == [0, 0, 1, 1, 0]


def test_sjoin_nearest(backend):
    pts, polys = _distance_frames()
    res = vs.sjoin_nearest(pts, polys, distance_col="dist")
    # (2, 0.5) ties: 1.0 from square 0 and from polygon 1
    got = sorted(zip(res.index, res["index_right"], res["dist"]))
    assert got == [(0, 0, 0.0), (1, 0, 1.0), (1, 1, 1.0), (2, 1, 0.5), (3, 0, 0.0), (4, 0, 5.0),
                   (5, 2, np.sqrt(8.0))]
    assert list(res.columns) == ["geometry", "qid", "index_right", "pid", "dist"]
    # max_distance: the far points drop out (inner) or keep NaN (left)
    inner = vs.sjoin_nearest(pts, polys, max_distance=1.0, distance_col="dist")
    assert sorted(set(inner.index)) == [0, 1, 2, 3]
    left = vs.sjoin_nearest(pts, polys, how="left", max_distance=1.0, distance_col="dist")
    # five matched rows (point 1 ties) + the two unmatched points
    assert left.shape[0] == 7 and np.isnan(left.loc[4, "dist"]) and np.isnan(left.loc[5, "index_right"])
    # how='right': the right frame's points get their nearest left polygons
    right = vs.sjoin_nearest(polys, pts, how="right", distance_col="dist")
    assert sorted(zip(right["index_left"], right.index)) == [(0, 0), (0, 1), (0, 3), (0, 4), (1, 1), (1, 2), (2, 5)]
    assert list(right.columns) == ["index_left", "pid", "geometry", "qid", "dist"]
    # polygons as the matched side: each polygon's nearest points (ties at 0 on square 0)
    rev = vs.sjoin_nearest(polys, pts, distance_col="dist")
    got = sorted(zip(rev.index, rev["index_right"], rev["dist"]))
    assert got == [(0, 0, 0.0), (0, 3, 0.0), (1, 2, 0.5), (2, 5, np.sqrt(8.0))]
    # and how='right' with the polygons on the right: the same query
    rr = vs.sjoin_nearest(pts, polys, how="right", distance_col="dist")
    assert sorted(zip(rr.index, rr["index_left"], rr["dist"])) == got
    with pytest.raises(NotImplementedError):
        vs.sjoin_nearest(pts, pts)
    with pytest.raises(ValueError):
        vs.sjoin_nearest(pts, polys, max_distance=-1)
    # the method form
    assert pts.sjoin_nearest(polys).shape == vs.sjoin_nearest(pts, polys).shape


def test_sjoin_nearest_cities_countries(backend):
    # tests/upstream/geopandas/tools/tests/test_sjoin.py:1355-1382: every city gets exactly one country,
    # inner == left, and max_distance=1 keeps exactly the rows with dist < 1
    w = dict(np.load(GOLDEN / "naturalearth_lowres.npz"))
    c = dict(np.load(GOLDEN / "naturalearth_cities.npz"))
    countries = vs.GeoDataFrame({"country": w["attr_name"]},
                                geometry=GeometryArray.from_polygon_buffers(w["x"], w["y"], w["ring_off"],
                                                                            w["part_off"], w["geom_off"],
                                                                            geom_type=w["geom_type"]))
    cities = vs.GeoDataFrame({"name": c["attr_name"]}, geometry=vs.points_from_xy(c["x"], c["y"]))
    r1 = vs.sjoin_nearest(cities, countries, distance_col="dist")
    assert r1.shape[0] == cities.shape[0]
    r3 = vs.sjoin_nearest(cities, countries, distance_col="dist", how="left")
    assert sorted(zip(r3.index, r3["index_right"])) == sorted(zip(r1.index, r1["index_right"]))
    r4 = vs.sjoin_nearest(cities, countries, distance_col="dist", max_distance=1)
    keep = r1[r1["dist"] < 1]
    assert sorted(zip(r4.index, r4["index_right"])) == sorted(zip(keep.index, keep["index_right"]))
    r5 = vs.sjoin_nearest(cities, countries, distance_col="dist", max_distance=1, how="left")
    assert r5.shape[0] == cities.shape[0]
    # cities inside their country are at distance 0 and agree with the within join
    within = vs.sjoin(cities, countries, predicate="within")
    zero = r1[r1["dist"] == 0]
    assert set(zip(within.index, within["index_right"])) <= set(zip(zero.index, zero["index_right"]))


def _sq(x, y, h=0.1):
    return vs.box(x - h, y - h, x + h, y + h)


def test_sjoin_nearest_empty_frames_and_max_distance(backend):
    """tests/upstream/geopandas/tools/tests/test_sjoin.py:1045-1176 (TestNearest),
    with small squares around the reference's right-hand points."""
    none = vs.GeoDataFrame({"geometry": GeometryArray.from_shapes([])})
    for kw in ({}, {"how": "inner"}, {"how": "left"}, {"how": "right"}):
        vs.sjoin_nearest(none, none, **kw)
    for how in ("outer", "abcde"):
        with pytest.raises(ValueError, match="`how` was"):
            vs.sjoin_nearest(none, none, how=how)
    pts = vs.GeoDataFrame({"geometry": [vs.Point(0, 0), vs.Point(1, 1)]})
    sqs = vs.GeoDataFrame({"geometry": [_sq(0, 0), _sq(1, 1)]})
    for col in (None, "distance"):
        j = vs.sjoin_nearest(pts, none, how="left", distance_col=col)
        assert len(j) == 2 and j["index_right"].isna().all()
        assert col is None or j[col].isna().all()
        j = vs.sjoin_nearest(pts, none, how="right", distance_col=col)
        assert j.empty and (col is None or col in j)
        for how in ("inner", "left"):
            j = vs.sjoin_nearest(none, sqs, how=how, distance_col=col)
            assert j.empty and (col is None or col in j)
        j = vs.sjoin_nearest(none, sqs, how="right", distance_col=col)
        assert len(j) == 2 and j["index_left"].isna().all()
        assert col is None or j[col].isna().all()
    # the join empties out under max_distance
    far = vs.GeoDataFrame({"geometry": [_sq(1, 1), _sq(2, 2)]})
    for how in ("inner", "left"):
        j = vs.sjoin_nearest(vs.GeoDataFrame({"geometry": [vs.Point(0, 0)]}), far, how=how, max_distance=1,
                             distance_col="distances")
        assert j.empty if how == "inner" else (j["index_right"].isna().all() and j["distances"].isna().all())
    # max_distance keeps the point inside a square, at distance 0
    for how in ("inner", "left"):
        j = vs.sjoin_nearest(pts, far, how=how, max_distance=1, distance_col="distances")
        if how == "inner":
            assert j.index.tolist() == [1] and j["index_right"].tolist() == [0] and j["distances"].tolist() == [0.0]
        else:
            assert np.isnan(j["index_right"].iloc[0]) and j["index_right"].iloc[1] == 0
            assert np.isnan(j["distances"].iloc[0]) and j["distances"].iloc[1] == 0.0


def test_attribute_codes_and_host_export():
    import importlib

    vs_sjoin = importlib.import_module("vibespatial_b200.sjoin")

    left = pd.DataFrame({"a": [1, 2, np.nan, 2, 3], "b": ["x", "y", "x", None, "y"]})
    right = pd.DataFrame({"a": [2, 1, 3, np.nan], "b": ["y", "x", "x", "x"]})
    lc, rc = vs_sjoin._attribute_codes(left, right, ["a"])
    # missing values never match; equal values share a code
    assert lc[2] == -1 and rc[3] == -1 and lc[1] == lc[3] == rc[0] and lc[0] == rc[1]
    lc2, rc2 = vs_sjoin._attribute_codes(left, right, ["a", "b"])
    assert lc2[3] == -1  # b missing
    assert lc2[1] == rc2[0] and lc2[0] == rc2[1] and lc2[4] != rc2[2]
    l = np.array([0, 0, 1, 3, 4, 4], np.intp)
    r = np.array([0, 1, 0, 0, 2, 3], np.intp)
    out_l, out_r, src = vs_sjoin._join_indexers(l, r, 5, 4, "left", (lc2, rc2))
    # kept pairs: (0,1) [x,1 == x,1], (1,0) [y,2 == y,2]; rows 2, 3, 4 unmatched
    assert out_l.tolist() == [0, 1, 2, 3, 4] and out_r.tolist() == [1, 0, -1, -1, -1]
    assert src.tolist() == [1, 2, -1, -1, -1]


def test_elementwise_distance_dwithin(backend):
    pts, polys = _distance_frames()
    p = pts.geometry.iloc[:3].reset_index(drop=True)
    g = polys.geometry.reset_index(drop=True)
    d = p.distance(g)
    # row-aligned: (0.5,0.5) in square 0; (2,0.5) 1 from polygon 1's edge x = 3; (4.5,1.5) vs box 2
    np.testing.assert_allclose(d.to_numpy(), [0.0, 1.0, np.hypot(5.5, 8.5)])
    assert p.dwithin(g, 1.0).tolist() == [True, True, False]
    assert p.dwithin(g, np.array([0.0, 0.5, 20.0])).tolist() == [True, False, True]
    # polygons on the left, a scalar point on the right, nulls
    assert g.distance(vs.Point(0.5, 0.5)).tolist()[0] == 0.0
    pn = vs.GeoSeries([None, vs.Point(0.5, 0.5), vs.Point(np.nan, 1.0)])
    dn = pn.distance(g)
    # row 1 pairs (0.5, 0.5) with polygon 1, whose left edge is x = 3
    assert np.isnan(dn[0]) and dn[1] == 2.5 and np.isnan(dn[2])
    assert pn.dwithin(g, 100.0).tolist() == [False, True, False]


def test_sindex_nearest(backend):
    pts, polys = _distance_frames()
    tree = polys.geometry.array
    q = pts.geometry.array
    idx, dist = tree.sindex.nearest(q, return_distance=True)
    assert idx[0].tolist() == [0, 1, 1, 2, 3, 4, 5] and idx[1].tolist() == [0, 0, 1, 1, 0, 0, 2]
    np.testing.assert_allclose(dist, [0, 1, 1, 0.5, 0, 5, np.sqrt(8)])
    one = tree.sindex.nearest(q, return_all=False)
    assert one[0].tolist() == [0, 1, 2, 3, 4, 5] and one[1].tolist() == [0, 0, 1, 0, 0, 2]
    assert tree.sindex.nearest(q, max_distance=0.6)[0].tolist() == [0, 2, 3]
    assert tree.sindex.nearest(vs.Point(8, 8)).tolist() == [[0], [2]]
    # polygons as the input, points as the tree
    r = q.sindex.nearest(tree)
    assert r[0].tolist() == [0, 0, 1, 2] and r[1].tolist() == [0, 3, 2, 5]
    with pytest.raises(NotImplementedError):
        tree.sindex.nearest(q, k=2)


def test_sindex_reductions(backend):
    tree = vs.GeometryArray.from_shapes([vs.box(0, 0, 5, 5), vs.box(3, 3, 6, 6), vs.box(10, 10, 11, 11)])
    q = vs.GeoSeries([vs.Point(1, 1), vs.Point(4, 4), vs.Point(20, 20)], index=["a", "b", "c"])
    anyhit = tree.sindex.query_any(q, predicate="intersects")
    assert anyhit.tolist() == [True, True, False] and list(anyhit.index) == ["a", "b", "c"]
    agg = tree.sindex.query_aggregate(q, {"n": "size", "w": (np.array([1.0, 10.0, 100.0]), "sum")},
                                      predicate="intersects")
    assert agg["n"].tolist() == [1, 2, 0] and agg["w"].tolist() == [1.0, 11.0, 0.0]
    assert tree.sindex.size == 3
    assert tree.sindex.intersection((4, 4)).tolist() == [0, 1]
    with pytest.raises(NotImplementedError):
        tree.sindex.intersection((0, 0, 1, 1))
    with pytest.raises(ValueError):
        tree.sindex.query_aggregate(q, {"n": "mean"})
    # validation of sindex._normalize_query_aggregations / _validate_query_aggregate_values
    with pytest.raises(ValueError, match="non-empty mapping"):
        tree.sindex.query_aggregate(q, {})
    with pytest.raises(TypeError, match="column names must be strings"):
        tree.sindex.query_aggregate(q, {1: "size"})
    with pytest.raises(ValueError, match="align with indexed tree geometries"):
        tree.sindex.query_aggregate(q, {"w": (np.array([1.0, 2.0]), "sum")})
    with pytest.raises(ValueError, match="one-dimensional"):
        tree.sindex.query_aggregate(q, {"w": (np.ones((3, 1)), "sum")})
    with pytest.raises(TypeError, match="must be numeric"):
        tree.sindex.query_aggregate(q, {"w": (np.array(["a", "b", "c"]), "sum")})


def test_sindex_relation_flow(backend):
    """query_relation, the semijoins, the antijoin, match counts, the pair
    aggregate of two aligned indexes and nearest_relation agree with the
    exported pairs of sindex.query / sindex.nearest."""
    tree = vs.GeometryArray.from_shapes([vs.box(0, 0, 5, 5), vs.box(3, 3, 6, 6), vs.box(10, 10, 11, 11),
                                         vs.box(30, 30, 31, 31)])
    q = vs.GeoSeries([vs.Point(1, 1), vs.Point(4, 4), vs.Point(20, 20), vs.Point(10.5, 10.5), vs.Point(4.5, 3.5)])
    rel = tree.sindex.query_relation(q, predicate="intersects")
    exported = tree.sindex.query(q, predicate="intersects")
    np.testing.assert_array_equal(rel.to_numpy(), exported)
    assert len(rel) == exported.shape[1] and rel.sorted_by_left
    assert rel.left_row_count == 5 and rel.right_row_count == 4
    host = tree.sindex.query_relation(q, predicate="intersects", return_device=False)
    assert not host.is_device
    np.testing.assert_array_equal(host.to_numpy(), exported)

    assert tree.sindex.query_left_semijoin(q, predicate="intersects").to_numpy().tolist() == [0, 1, 3, 4]
    assert tree.sindex.query_left_antijoin(q, predicate="intersects").to_numpy().tolist() == [2]
    assert tree.sindex.query_right_semijoin(q, predicate="intersects").to_numpy().tolist() == [0, 1, 2]
    counts = tree.sindex.query_left_match_count_expression(q, predicate="intersects")
    assert counts.to_numpy().tolist() == [1, 2, 0, 1, 2] and counts.source_row_count == 5
    assert counts.compare_scalar_selection(">", 1).to_numpy().tolist() == [1, 4]
    with pytest.raises(ValueError):
        counts.compare_scalar_selection("~", 1)

    # a second index aligned with the first: row 0 smaller, row 1 the same, rows 2-3 elsewhere
    other = vs.GeometryArray.from_shapes([vs.box(0, 0, 2, 2), vs.box(3, 3, 6, 6), vs.box(50, 50, 51, 51),
                                          vs.box(10, 10, 11, 11)])
    agg = tree.sindex.query_pair_aggregate(other.sindex, q, predicate="intersects")
    assert list(agg.columns) == ["left_count", "right_count", "shared_count"]
    assert agg["left_count"].tolist() == [3, 2, 1, 0]
    assert agg["right_count"].tolist() == [1, 2, 0, 1]
    assert agg["shared_count"].tolist() == [1, 2, 0, 0]
    with pytest.raises(TypeError):
        tree.sindex.query_pair_aggregate(object(), q, predicate="intersects")
    with pytest.raises(ValueError, match="equal size"):
        tree.sindex.query_pair_aggregate(vs.GeometryArray.from_shapes([vs.box(0, 0, 1, 1)]).sindex, q)

    # dwithin: (20, 20) is 12.73 from the third box and 14.14 from the fourth
    assert tree.sindex.query_left_semijoin(q, predicate="dwithin", distance=10.0).to_numpy().tolist() == [0, 1, 3, 4]
    assert tree.sindex.query_left_semijoin(q, predicate="dwithin", distance=13.0).to_numpy().tolist() == [0, 1, 2, 3,
                                                                                                        4]
    assert tree.sindex.query_right_semijoin(q, predicate="dwithin", distance=13.0).to_numpy().tolist() == [0, 1, 2]
    counts = tree.sindex.query_left_match_count_expression(q, predicate="dwithin", distance=13.0)
    assert counts.to_numpy().tolist() == [3, 3, 1, 3, 3]  # at 13 every point but (20, 20) reaches three boxes

    near = tree.sindex.nearest_relation(q)
    pairs, dist = tree.sindex.nearest(q, return_distance=True)
    np.testing.assert_array_equal(near.to_numpy(), pairs)
    np.testing.assert_array_equal(near.distances, dist)
    assert near.predicate == "nearest"
