"""Bit-exact pair sets at the full sizes of the benchmark configurations.

Each workload is generated once per module and joined once by the CPU oracle
per predicate; every CUDA path that runs the workload (the plain R-tree, the
learned single join, the batch plans with graph replay) must give exactly
the oracle's sorted (point row, polygon row) pairs.

* degenerate: 20M points x 200k polygons with 1-5 holes, 2-4-part
  multipolygons, 10% of the points on vertices, 10% on edges (dyadic t),
  10% one ulp off edges; within / intersects, and contains with the polygons
  as the input side through query_spatial_index (the reference evaluates
  contains as the swapped within, src/vibespatial/api/tools/sjoin.py:1052-1082;
  near-edge traps as in tests/test_point_in_polygon.py:135-190)
* utm: 10M points x 100k footprints, intersects (within is in test_gpu_parity)
* batched: all 256 jobs, learned and R-tree batch plans replayed from a graph
* zipf: 50M points x 1M footprints through the one-job learned batch plan the
  benchmark times, the learned single join and the plain R-tree
"""
from types import SimpleNamespace

import numpy as np
import pytest

from _helpers import PRED_CODES, assert_same_pairs, oracle_polys, upload_points, upload_polys

pytestmark = pytest.mark.gpu


def _sorted_np(vsabi, ctx, left, right):
    """Device pairs sorted by (left, right) on the device, as int64 host arrays."""
    if left.numel():
        vsabi.sort_pairs(ctx, left, right)
    return left.cpu().numpy().astype(np.int64), right.cpu().numpy().astype(np.int64)


# ----------------------------------------------------------- degenerate ---

@pytest.fixture(scope="module")
def degenerate(vsabi, ctx, oracle):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.degenerate_join(seed=5)  # 20M x 200k
    P, keep_p = upload_polys(vsabi, w.polys)
    pts, keep_q = upload_points(vsabi, w.px, w.py)
    index = vsabi.DeviceIndex(ctx, P, learned=True)
    OP = oracle_polys(oracle, w.polys)
    exp = {p: oracle.join(w.px, w.py, None, OP, p) for p in ("within", "intersects")}
    return SimpleNamespace(w=w, index=index, pts=pts, exp=exp, keep=(keep_p, keep_q))


def test_degenerate_cell_level_is_refined(degenerate):
    """The multipolygons' wide boxes pull the mean box side up (level 7 from it, 35 entries per cell); the automatic
    level is refined while an entry's cell holds more than 2.5 entries on average, within the registration budget
    (level 10 would exceed it).  260k cell keys keep the default 4096 RMI leaves."""
    info = degenerate.index.info()
    assert info["cell_level"] >= 8
    assert info["n_cell_entries"] / info["n_cells"] < 12.0
    assert info["rmi_leaves"] == 4096


@pytest.mark.parametrize("method", ["rtree", "learned"])
@pytest.mark.parametrize("predicate", ["within", "intersects"])
def test_degenerate_full_size(vsabi, degenerate, predicate, method):
    d = degenerate
    m = vsabi.METHOD_RTREE if method == "rtree" else vsabi.METHOD_LEARNED
    gl, gr, st = d.index.join(d.pts, PRED_CODES[predicate], m, sort=True)
    el, er = d.exp[predicate]
    assert_same_pairs(gl.cpu().numpy(), gr.cpu().numpy(), el, er)
    if predicate == "intersects":
        assert st["exact_fallbacks"] > 0  # on-edge points reach the exact stage
    if method == "learned":
        assert st["fp32_edges"] > 0 and st["fp64_edges"] > 0


@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_degenerate_full_size_contains(degenerate, method):
    """contains(polygon, point) with the polygons as the input side: the swapped within pairs."""
    from vibespatial_b200.geometry import GeometryArray
    from vibespatial_b200.query import query_spatial_index

    w = degenerate.w
    tree = GeometryArray.from_points(w.px, w.py)
    geom = GeometryArray.from_polygon_buffers(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off,
                                              w.polys.geom_off)
    out = query_spatial_index(tree, geom, predicate="contains", method=method)
    el, er = degenerate.exp["within"]
    o = np.lexsort((el, er))
    assert out.shape == (2, len(el))
    np.testing.assert_array_equal(out[0], er[o])
    np.testing.assert_array_equal(out[1], el[o])


def test_degenerate_full_size_batch_plan(vsabi, ctx, degenerate):
    """The degenerate workload as a one-job learned batch plan replayed from a graph (grows its deferred buffer)."""
    d = degenerate
    plan = vsabi.BatchPlan(ctx, [d.index], d.pts, [0, d.w.n_points], options={"method": vsabi.METHOD_LEARNED})
    for predicate in ("within", "intersects"):
        left, right, _ = plan.run(PRED_CODES[predicate], use_graph=True)
        gl, gr = _sorted_np(vsabi, ctx, left, right)
        assert_same_pairs(gl, gr, *d.exp[predicate])


# ------------------------------------------------------------------ utm ---

@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_full_size_utm_intersects(vsabi, ctx, oracle, method):
    """The UTM-frame workload at full size (10M x 100k), intersects."""
    from _helpers import gpu_join
    from vibespatial_b200.testing import synthetic as syn

    w = syn.utm_join(seed=1)
    el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "intersects")
    gl, gr, _ = gpu_join(vsabi, ctx, w.px, w.py, w.polys, "intersects",
                         vsabi.METHOD_RTREE if method == "rtree" else vsabi.METHOD_LEARNED)
    assert_same_pairs(gl, gr, el, er)


# -------------------------------------------------------------- batched ---

@pytest.fixture(scope="module")
def batched256(vsabi, ctx, oracle):
    from vibespatial_b200.testing import synthetic as syn

    jobs = syn.batched_jobs(seed=2, n_jobs=256)  # the benchmark's 256 jobs (69.6M points)
    px = np.concatenate([w.px for w in jobs])
    py = np.concatenate([w.py for w in jobs])
    job_start = np.concatenate([[0], np.cumsum([w.n_points for w in jobs])]).astype(np.int64)
    pts, keep_q = upload_points(vsabi, px, py)
    indexes, keep = [], [keep_q]
    for w in jobs:
        P, bufs = upload_polys(vsabi, w.polys)
        keep.append(bufs)
        indexes.append(vsabi.DeviceIndex(ctx, P, learned=True))
    exp = [oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "within") for w in jobs]
    return SimpleNamespace(jobs=jobs, job_start=job_start, pts=pts, indexes=indexes, exp=exp, keep=keep)


@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_batched_256_jobs_full_size(vsabi, ctx, batched256, method):
    """Every one of the 256 jobs: pairs equal the oracle's for that job alone, graph captured then replayed."""
    b = batched256
    opts = {"method": vsabi.METHOD_LEARNED} if method == "learned" else None
    plan = vsabi.BatchPlan(ctx, b.indexes, b.pts, b.job_start, options=opts)
    for rep in range(2):  # capture, then replay
        left, right, _ = plan.run(PRED_CODES["within"], use_graph=True)
        gl, gr = _sorted_np(vsabi, ctx, left, right)
        job = np.searchsorted(b.job_start, gl, side="right") - 1
        bounds = np.searchsorted(job, np.arange(len(b.jobs) + 1))
        for j in range(len(b.jobs)):
            s = slice(bounds[j], bounds[j + 1])
            el, er = b.exp[j]
            assert_same_pairs(gl[s] - b.job_start[j], gr[s], el, er)


# ----------------------------------------------------------------- zipf ---

@pytest.fixture(scope="module")
def zipf(vsabi, ctx, oracle):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.zipf_join(seed=3)  # 50M x 1M, the benchmark's default workload
    P, keep_p = upload_polys(vsabi, w.polys)
    pts, keep_q = upload_points(vsabi, w.px, w.py)
    index = vsabi.DeviceIndex(ctx, P, learned=True)
    exp = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "within")
    return SimpleNamespace(w=w, index=index, pts=pts, exp=exp, keep=(keep_p, keep_q))


def test_zipf_cell_level_follows_the_dense_cells(zipf):
    """Zipf's clusters: the plain mean is 1.55 entries per cell at level 12, but an entry's cell holds 3.3 on
    average, so the automatic level goes to 13 (2.4); its 5.5M cell keys get one RMI leaf per 64 keys, capped at
    65535, which keeps the error windows a few dozen keys wide (432 with 4096 leaves)."""
    info = zipf.index.info()
    assert info["cell_level"] == 13
    assert info["rmi_leaves"] == 65535
    assert info["rmi_mean_window"] < 60


@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_full_size_zipf_join(vsabi, zipf, method):
    """50M x 1M, within: the plain R-tree and the learned single join give the oracle's pairs."""
    m = vsabi.METHOD_RTREE if method == "rtree" else vsabi.METHOD_LEARNED
    gl, gr, _ = zipf.index.join(zipf.pts, PRED_CODES["within"], m, sort=True)
    assert_same_pairs(gl.cpu().numpy(), gr.cpu().numpy(), *zipf.exp)


def test_full_size_zipf_benchmarked_plan(vsabi, ctx, zipf):
    """50M x 1M, within, through the exact call the benchmark times: a one-job learned batch plan
    replayed from a CUDA graph into preallocated buffers (first call captures, later calls replay)."""
    import torch

    n = zipf.w.n_points
    plan = vsabi.BatchPlan(ctx, [zipf.index], zipf.pts, [0, n], options={"method": vsabi.METHOD_LEARNED})
    cap = max(1024, n)
    left = torch.empty(cap, dtype=torch.int32, device="cuda")
    right = torch.empty(cap, dtype=torch.int32, device="cuda")
    for _ in range(3):
        k, _st = plan.run_into(PRED_CODES["within"], left, right, use_graph=True)
        gl, gr = _sorted_np(vsabi, ctx, left[:k].clone(), right[:k].clone())
        assert_same_pairs(gl, gr, *zipf.exp)
