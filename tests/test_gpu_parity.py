"""CUDA join parity against the exact CPU oracle (bit-exact pair sets).

Every test calls through the C-ABI (libvsjoin.so via ctypes) and compares
with oracle/ on the same seeded inputs.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import _shapes as S
from _helpers import PRED_CODES, assert_same_pairs, gpu_join, oracle_polys, to_dev, upload_points, upload_polys

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
METHODS = {"rtree": 0, "learned": 1, "brute": 2}


def _check(vsabi, ctx, oracle, w, predicate, method=0, pvalid=None):
    P = oracle_polys(oracle, w.polys)
    el, er = oracle.join(w.px, w.py, pvalid, P, predicate)
    gl, gr, stats = gpu_join(vsabi, ctx, w.px, w.py, w.polys, predicate, method, pvalid)
    assert_same_pairs(gl, gr, el, er)
    return stats


@pytest.mark.parametrize("predicate", ["within", "intersects", "covered_by", "touches", None])
@pytest.mark.parametrize("method", ["rtree", "learned", "brute"])
def test_star_join_all_predicates(vsabi, ctx, oracle, predicate, method):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=0)  # 100k points x 1k star polygons
    _check(vsabi, ctx, oracle, w, predicate, METHODS[method])


@pytest.mark.parametrize("method", ["rtree", "learned"])
@pytest.mark.parametrize("predicate", ["within", "intersects"])
def test_utm_join_reduced(vsabi, ctx, oracle, predicate, method):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.utm_join(seed=1, n_points=1_000_000, n_polys=100_000)
    stats = _check(vsabi, ctx, oracle, w, predicate, METHODS[method])
    if method == "learned":
        assert stats["fp32_edges"] > 0


@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_zipf_join_reduced(vsabi, ctx, oracle, method):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.zipf_join(seed=3, n_points=2_000_000, n_polys=100_000)
    _check(vsabi, ctx, oracle, w, "within", METHODS[method])


@pytest.mark.parametrize("method", ["rtree", "learned"])
@pytest.mark.parametrize("predicate", ["within", "intersects", "touches"])
def test_degenerate_join_reduced(vsabi, ctx, oracle, predicate, method):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.degenerate_join(seed=5, n_points=400_000, n_polys=4_000)
    stats = _check(vsabi, ctx, oracle, w, predicate, METHODS[method])
    if predicate != "within":
        assert stats["exact_fallbacks"] > 0  # on-edge points must reach the exact stage
    if method == "learned":
        assert stats["fp64_edges"] > 0  # near-boundary edges leave the FP32 filter


@pytest.mark.parametrize("workload", ["star", "zipf", "degenerate"])
def test_rtree_bulk_leaf_copies(vsabi, ctx, oracle, workload):
    """The plain traversal with leaf blocks loaded by bulk copies (TMA) gives the oracle's pairs."""
    from vibespatial_b200.testing import synthetic as syn

    w = {"star": lambda: syn.star_join(seed=0),
         "zipf": lambda: syn.zipf_join(seed=3, n_points=2_000_000, n_polys=100_000),
         "degenerate": lambda: syn.degenerate_join(seed=5, n_points=200_000, n_polys=3_000)}[workload]()
    for predicate in ("within", "intersects"):
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), predicate)
        pts, _k1 = upload_points(vsabi, w.px, w.py)
        P, _k2 = upload_polys(vsabi, w.polys)
        index = vsabi.DeviceIndex(ctx, P)
        gl, gr, _ = index.join(pts, PRED_CODES[predicate], vsabi.METHOD_RTREE, flags=vsabi.JOIN_BULK_LEAVES)
        assert_same_pairs(gl.cpu().numpy(), gr.cpu().numpy(), el, er)


@pytest.mark.parametrize("bin_min", [4, -1])
@pytest.mark.parametrize("workload", ["star", "degenerate"])
def test_ring_bins(vsabi, ctx, oracle, workload, bin_min):
    """Walking only a point's y-bin of edges (bins on every ring of >= 4 vertices) or every edge (no bins)
    gives the oracle's pairs for every method, on boundary and 1-ulp points too."""
    from vibespatial_b200.testing import synthetic as syn

    w = (syn.star_join(seed=2, n_points=100_000, n_polys=2_000) if workload == "star"
         else syn.degenerate_join(seed=8, n_points=200_000, n_polys=3_000))
    pts, _k1 = upload_points(vsabi, w.px, w.py)
    P, _k2 = upload_polys(vsabi, w.polys)
    index = vsabi.DeviceIndex(ctx, P, learned=True, ring_bin_min_vertices=bin_min)
    info = index.info()
    assert (info["n_binned_rings"] > 0) == (bin_min > 0)
    for predicate in ("within", "intersects", "touches"):
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), predicate)
        for method in (vsabi.METHOD_RTREE, vsabi.METHOD_LEARNED, vsabi.METHOD_BRUTE):
            gl, gr, _ = index.join(pts, PRED_CODES[predicate], method)
            assert_same_pairs(gl.cpu().numpy(), gr.cpu().numpy(), el, er)


def test_learned_index_agrees_with_rtree(vsabi, ctx):
    """Learned lookups and plain traversal give the same pair set (the R-tree is the arbiter)."""
    from vibespatial_b200.testing import synthetic as syn

    w = syn.zipf_join(seed=13, n_points=3_000_000, n_polys=200_000)
    P, keep = upload_polys(vsabi, w.polys)
    index = vsabi.DeviceIndex(ctx, P, learned=True)
    info = index.info()
    assert info["n_cells"] > 0 and info["rmi_max_window"] >= 1
    for pred in ("within", "intersects", None):
        al, ar, _ = gpu_join(vsabi, ctx, w.px, w.py, None, pred, 0, index=index)
        bl, br, st = gpu_join(vsabi, ctx, w.px, w.py, None, pred, 1, index=index)
        assert_same_pairs(bl, br, al, ar)
    # explicit grid levels, including very coarse and very fine ones
    for level in (3, 9, 15):
        idx2 = vsabi.DeviceIndex(ctx, P, learned=True, cell_level=level, rmi_leaves=512, rmi_train_steps=50)
        bl, br, _ = gpu_join(vsabi, ctx, w.px[:500_000], w.py[:500_000], None, "within", 1, index=idx2)
        al, ar, _ = gpu_join(vsabi, ctx, w.px[:500_000], w.py[:500_000], None, "within", 0, index=idx2)
        assert_same_pairs(bl, br, al, ar)


@pytest.mark.parametrize("name", sorted(S.KNOWN_COVERS))
def test_known_cases_aligned(vsabi, ctx, oracle, name):
    polys, pts, expected = S.KNOWN_COVERS[name]
    P = S.soa(polys)
    px, py, pv = S.points(pts)
    exp = oracle.locate_aligned(px, py, pv, oracle.Polygons(P.x, P.y, P.ring_off, P.part_off, P.geom_off, P.valid))
    dpts, k1 = upload_points(vsabi, px, py, pv)
    dpol, k2 = upload_polys(vsabi, P)
    import torch

    out = torch.empty(len(px), dtype=torch.uint8, device="cuda")
    vsabi.locate_aligned(ctx, dpts, dpol, out)
    np.testing.assert_array_equal(out.cpu().numpy(), exp)


def test_known_cases_join(vsabi, ctx, oracle):
    tree, pts, (el, er) = S.SPATIAL_QUERY_CASE
    P = S.soa(tree)
    px, py, _ = S.points(pts)
    gl, gr, _ = gpu_join(vsabi, ctx, px, py, P, "intersects")
    assert gl.tolist() == el and gr.tolist() == er


@pytest.mark.parametrize("method", [0, 1])
def test_nybb_and_natural_earth(vsabi, ctx, oracle, method):
    from test_oracle_golden import nybb_points

    exp = json.loads((GOLDEN / "expected.json").read_text())
    d = dict(np.load(GOLDEN / "nybb.npz"))
    P, px, py = nybb_points(d, oracle)
    poly = S.SoA(d["x"], d["y"], d["ring_off"], d["part_off"], d["geom_off"], np.ones(len(d["geom_off"]) - 1))
    gl, gr, _ = gpu_join(vsabi, ctx, px, py, poly, "intersects", method)
    assert len(gl) == exp["nybb_inner_intersects_shape"]["value"][0]
    el, er = oracle.join(px, py, None, P, "intersects")
    assert_same_pairs(gl, gr, el, er)
    w = dict(np.load(GOLDEN / "naturalearth_lowres.npz"))
    c = dict(np.load(GOLDEN / "naturalearth_cities.npz"))
    wp = S.SoA(w["x"], w["y"], w["ring_off"], w["part_off"], w["geom_off"], np.ones(len(w["geom_off"]) - 1))
    gl, gr, _ = gpu_join(vsabi, ctx, c["x"], c["y"], wp, "intersects", method)
    assert len(gl) == exp["cities_countries_inner_intersects_shape"]["value"][0]


@pytest.mark.parametrize("method", [0, 1])
def test_edge_cases(vsabi, ctx, oracle, method):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=4, n_points=5000, n_polys=50)
    # empty point set
    gl, gr, _ = gpu_join(vsabi, ctx, w.px[:0], w.py[:0], w.polys, "within", method)
    assert len(gl) == 0
    # empty polygon set
    empty = S.soa([])
    gl, gr, _ = gpu_join(vsabi, ctx, w.px, w.py, empty, "within", method)
    assert len(gl) == 0
    # one polygon (the root is the only item)
    one = S.soa([S.box(100, 100, 900, 900)])
    gl, gr, _ = gpu_join(vsabi, ctx, w.px, w.py, one, "intersects", method)
    el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, one), "intersects")
    assert_same_pairs(gl, gr, el, er)
    # null / NaN points and null / empty polygons never match
    px, py = w.px.copy(), w.py.copy()
    pv = np.ones(len(px), np.uint8)
    pv[::7] = 0
    px[::11] = np.nan
    gl, gr, _ = gpu_join(vsabi, ctx, px, py, w.polys, "intersects", method, pvalid=pv)
    el, er = oracle.join(px, py, pv, oracle_polys(oracle, w.polys), "intersects")
    assert_same_pairs(gl, gr, el, er)
    mixed = S.soa([None, [], S.box(0, 0, 500, 500), None, S.box(400, 400, 1000, 1000)])
    gl, gr, _ = gpu_join(vsabi, ctx, w.px, w.py, mixed, "within", method)
    el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, mixed), "within")
    assert_same_pairs(gl, gr, el, er)
    assert set(np.unique(gr)) <= {2, 4}


@pytest.mark.parametrize("method", ["rtree", "learned", "brute"])
def test_last_hilbert_cell_with_null_points(vsabi, ctx, oracle, method):
    """Valid points in the frame's last Hilbert cell (the corner (maxx, miny))
    sort before every null point even though the sort orders only the top key
    bits; null points there never match."""
    polys = S.soa([S.box(0, 0, 1000, 1000), S.box(990, 0, 1000, 10), S.box(0, 990, 10, 1000)])
    rng = np.random.default_rng(3)
    k = 4000
    # half the points inside the last level-12 cell of the frame, interleaved with null points
    px = np.concatenate([1000 - rng.uniform(0, 0.2, k), rng.uniform(0, 1000, k)])
    py = np.concatenate([rng.uniform(0, 0.2, k), rng.uniform(0, 1000, k)])
    pv = (np.arange(2 * k) % 3 != 0).astype(np.uint8)
    P = oracle_polys(oracle, polys)
    for predicate in ("intersects", "within"):
        el, er = oracle.join(px, py, pv, P, predicate)
        gl, gr, _ = gpu_join(vsabi, ctx, px, py, polys, predicate, METHODS[method], pv)
        assert_same_pairs(gl, gr, el, er)


def test_index_counts_skip_null_polygons(vsabi, ctx, oracle):
    """Null polygons own no rings in the index's layout; later passes over
    the layout (the ring y-bins, the learned index's FP32 vertices) cover only
    the laid-out rings."""
    from types import SimpleNamespace

    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=6, n_points=20_000, n_polys=400)  # 8-64 vertices: long rings get y-bins
    m = len(w.polys.geom_off) - 1
    gvalid = (np.arange(m) % 3 != 0).astype(np.uint8)
    polys = SimpleNamespace(x=w.polys.x, y=w.polys.y, ring_off=w.polys.ring_off, part_off=w.polys.part_off,
                            geom_off=w.polys.geom_off, valid=gvalid)
    pts, keep1 = upload_points(vsabi, w.px, w.py, None)
    P, keep2 = upload_polys(vsabi, polys)
    index = vsabi.DeviceIndex(ctx, P, learned=True)
    info = index.info()
    n_valid_rings = int(gvalid.sum())  # one ring per star polygon
    assert 0 < info["n_binned_rings"] <= n_valid_rings
    el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, polys), "within")
    for method in (0, 1):
        gl, gr, _ = index.join(pts, PRED_CODES["within"], method, sort=True)
        assert_same_pairs(gl.cpu().numpy(), gr.cpu().numpy(), el, er)


def test_capacity_error_reports_required_size(vsabi, ctx, oracle):
    import torch
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=0)
    el, _ = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "within")
    dpts, k1 = upload_points(vsabi, w.px, w.py)
    dpol, k2 = upload_polys(vsabi, w.polys)
    index = vsabi.DeviceIndex(ctx, dpol)
    small = torch.empty(100, dtype=torch.int32, device="cuda")
    small2 = torch.empty(100, dtype=torch.int32, device="cuda")
    with pytest.raises(vsabi.CapacityError) as ei:
        index.join_into(dpts, PRED_CODES["within"], 0, small, small2)
    assert ei.value.required == len(el)
    # bad arguments are rejected before any launch
    with pytest.raises(ValueError):
        index.join_into(dpts, 99, 0, small, small2)


def test_radix_sort_and_hilbert_keys(vsabi, ctx):
    import torch

    rng = np.random.default_rng(9)
    for n, bits in [(1, 64), (4095, 64), (4097, 24), (300_000, 64), (1_000_003, 40)]:
        keys = rng.integers(0, 2**63, n, dtype=np.int64).view(np.uint64) >> np.uint64(64 - bits)
        keys[::3] = keys[0]  # duplicates: stability check
        vals = np.arange(n, dtype=np.uint32)
        dk = torch.from_numpy(keys.view(np.int64)).cuda()
        dv = torch.from_numpy(vals.view(np.int32)).cuda()
        vsabi.radix_sort_pairs(ctx, dk, dv, bits)
        order = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
        np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])
    x = rng.uniform(0, 10, 1000)
    y = rng.uniform(0, 10, 1000)
    out = torch.empty(1000, dtype=torch.int64, device="cuda")
    vsabi.hilbert_keys(ctx, to_dev(x), to_dev(y), (0, 0, 10, 10), out)
    got = out.cpu().numpy().view(np.uint64)
    sc = 4294967295.0 / 10
    exp = [vsabi.hilbert_key_host(min(int(a * sc), 0xFFFFFFFF), min(int(b * sc), 0xFFFFFFFF)) for a, b in zip(x, y)]
    np.testing.assert_array_equal(got, np.array(exp, dtype=np.uint64))


def test_pair_sort(vsabi, ctx):
    import torch

    rng = np.random.default_rng(1)
    l = rng.integers(0, 1 << 30, 200_000).astype(np.int32)
    r = rng.integers(0, 1 << 30, 200_000).astype(np.int32)
    dl, dr = torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()
    vsabi.sort_pairs(ctx, dl, dr)
    o = np.lexsort((r, l))
    np.testing.assert_array_equal(dl.cpu().numpy(), l[o])
    np.testing.assert_array_equal(dr.cpu().numpy(), r[o])


@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_full_size_utm_join(vsabi, ctx, oracle, method):
    """The UTM-frame workload at full size (10M x 100k), within: whole pair set equal."""
    from vibespatial_b200.testing import synthetic as syn

    w = syn.utm_join(seed=1)
    _check(vsabi, ctx, oracle, w, "within", METHODS[method])


@pytest.mark.parametrize("chunk", [None, 3_000_000])
@pytest.mark.parametrize("method", ["rtree", "learned"])
def test_join_host_pipeline(vsabi, ctx, oracle, method, chunk, monkeypatch):
    """vs_join_host (chunked host->device->host pipeline) gives the oracle's pairs: one or several
    chunks, a null mask, sorted and unsorted output, and the capacity error."""
    import torch

    from vibespatial_b200.testing import synthetic as syn

    if chunk:
        monkeypatch.setenv("VSJOIN_HOST_CHUNK", str(chunk))  # 3 chunks
    w = syn.zipf_join(seed=12, n_points=9_000_000, n_polys=150_000)
    rng = np.random.default_rng(1)
    pvalid = (rng.random(w.n_points) > 0.05).astype(np.uint8)
    P, _k = upload_polys(vsabi, w.polys)
    index = vsabi.DeviceIndex(ctx, P, learned=True)
    el, er = oracle.join(w.px, w.py, pvalid, oracle_polys(oracle, w.polys), "intersects")
    hx = torch.from_numpy(w.px).pin_memory()
    hy = torch.from_numpy(w.py).pin_memory()
    hv = torch.from_numpy(pvalid).pin_memory()
    cap = len(el) + 100
    hl = torch.empty(cap, dtype=torch.int32).pin_memory()
    hr = torch.empty(cap, dtype=torch.int32).pin_memory()
    m = METHODS[method]
    n, _ = index.join_host(hx, hy, PRED_CODES["intersects"], m, hl, hr, valid=hv, sort=True)
    assert_same_pairs(hl[:n].numpy(), hr[:n].numpy(), el, er)
    n2, _ = index.join_host(w.px, w.py, PRED_CODES["intersects"], m, hl.numpy(), hr.numpy(), valid=pvalid)
    l2, r2 = hl[:n2].numpy(), hr[:n2].numpy()
    o = np.lexsort((r2, l2))
    assert_same_pairs(l2[o], r2[o], el, er)
    with pytest.raises(vsabi.CapacityError) as ei:
        index.join_host(hx, hy, PRED_CODES["intersects"], m, hl[:10], hr[:10], valid=hv)
    assert ei.value.required == len(el)


def test_join_host_grows_chunk_pair_buffer(vsabi, ctx, oracle):
    """More pairs than points: the chunk's pair buffer grows and the chunk reruns."""
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=13, n_points=300_000, n_polys=20_000)  # several box candidates per point
    P, _k = upload_polys(vsabi, w.polys)
    index = vsabi.DeviceIndex(ctx, P)
    for predicate in (None, "intersects"):
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), predicate)
        hl = np.empty(len(el), np.int32)
        hr = np.empty(len(el), np.int32)
        n, _ = index.join_host(w.px, w.py, PRED_CODES[predicate], vsabi.METHOD_RTREE, hl, hr, sort=True)
        assert n == len(el) > w.n_points  # more pairs than the first chunk buffer holds
        assert_same_pairs(hl, hr, el, er)


@pytest.mark.parametrize("flags", ["bsearch", "fp64_walk", "both", "no_stage", "no_interior"])
@pytest.mark.parametrize("workload", ["zipf", "degenerate"])
def test_learned_ablation_switches(vsabi, ctx, oracle, workload, flags):
    """The learned method with its RMI replaced by a binary search over every cell key, with FP64 ring walks
    instead of the FP32 stage, without the bulk-copy staging of candidate records or without the interior-box
    shortcut (the ablations the benchmark times) still gives the oracle's pairs."""
    from vibespatial_b200.testing import synthetic as syn

    w = (syn.zipf_join(seed=14, n_points=1_000_000, n_polys=50_000) if workload == "zipf"
         else syn.degenerate_join(seed=15, n_points=300_000, n_polys=3_000))
    f = {"bsearch": vsabi.JOIN_LEARNED_BSEARCH, "fp64_walk": vsabi.JOIN_LEARNED_FP64_WALK,
         "both": vsabi.JOIN_LEARNED_BSEARCH | vsabi.JOIN_LEARNED_FP64_WALK,
         "no_stage": vsabi.JOIN_LEARNED_NO_STAGE, "no_interior": vsabi.JOIN_LEARNED_NO_INTERIOR}[flags]
    pts, _k1 = upload_points(vsabi, w.px, w.py)
    P, _k2 = upload_polys(vsabi, w.polys)
    index = vsabi.DeviceIndex(ctx, P, learned=True)
    for predicate in ("within", "intersects"):
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), predicate)
        gl, gr, st = index.join(pts, PRED_CODES[predicate], vsabi.METHOD_LEARNED, flags=f)
        assert_same_pairs(gl.cpu().numpy(), gr.cpu().numpy(), el, er)
        if f & vsabi.JOIN_LEARNED_FP64_WALK:
            assert st["fp32_edges"] == 0
        if f & vsabi.JOIN_LEARNED_BSEARCH:
            assert st["rmi_fallbacks"] == 0
