"""Distance joins on the GPU (vs_join_dwithin, vs_join_nearest) against the
CPU oracle: bit-exact pair sets and bit-exact distances.

Workloads: star polygons, holes + multipolygons with on-edge / on-vertex /
1-ulp points, a lattice of squares sharing edges (ties), points far outside
the polygon frame, null and NaN points, null polygons; scalar, per-point
and per-polygon distances including 0, negative and NaN; bounded and
unbounded nearest searches; the capacity error path.
"""
import numpy as np
import pytest

from vibespatial_b200.testing import synthetic as syn

pytestmark = pytest.mark.gpu


def _device(vsabi, ctx, w, *, pvalid=None, gvalid=None, learned=False):
    import torch

    p = w.polys
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k))).cuda()
         for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    gv = None if gvalid is None else torch.from_numpy(gvalid.astype(np.uint8)).cuda()
    P = vsabi.make_polygons(t["x"], t["y"], t["ring_off"], t["part_off"], t["geom_off"], gv)
    index = vsabi.DeviceIndex(ctx, P, learned=learned)
    dx = torch.from_numpy(np.ascontiguousarray(w.px)).cuda()
    dy = torch.from_numpy(np.ascontiguousarray(w.py)).cuda()
    pv = None if pvalid is None else torch.from_numpy(pvalid.astype(np.uint8)).cuda()
    pts = vsabi.make_points(dx, dy, pv)
    return index, pts, (t, gv, dx, dy, pv)


def _oracle_polys(oracle, w, gvalid=None):
    p = w.polys
    return oracle.Polygons(p.x, p.y, p.ring_off, p.part_off, p.geom_off, gvalid)


def _with_outside_points(w, rng, k=64):
    """Append points far outside the polygon frame, NaN points and infinities."""
    lo, hi = float(np.min(w.polys.x)), float(np.max(w.polys.x))
    span = hi - lo
    ox = np.concatenate([rng.uniform(lo - 3 * span, lo - span, k // 2), rng.uniform(hi + span, hi + 2 * span, k // 2)])
    oy = rng.uniform(lo - span, hi + span, k)
    px = np.concatenate([w.px, ox, [np.nan, 1.0, np.inf]])
    py = np.concatenate([w.py, oy, [1.0, np.nan, 0.0]])
    return syn.Workload(name=w.name + "+outside", px=px, py=py, polys=w.polys)


def _lattice(n=12):
    """n x n unit squares sharing edges; points on lattice lines, at vertices and at centres (ties)."""
    rings = []
    for i in range(n):
        for j in range(n):
            rings.append(np.array([(i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1), (i, j)], float))
    sizes = np.array([len(r) for r in rings])
    xs = np.concatenate([r[:, 0] for r in rings])
    ys = np.concatenate([r[:, 1] for r in rings])
    polys = syn._rings_to_soa(sizes, xs, ys)
    g = np.arange(0, n + 0.5, 0.5)
    gx, gy = np.meshgrid(g, g)
    px = np.concatenate([gx.ravel(), [-1.5, n + 2.0, n / 2.0]])
    py = np.concatenate([gy.ravel(), [-1.5, n / 2.0, -0.75]])
    return syn.Workload(name="lattice", px=px, py=py, polys=polys)


WORKLOADS = {
    "star": lambda: syn.star_join(seed=11, n_points=20_000, n_polys=300),
    "degenerate": lambda: syn.degenerate_join(seed=12, n_points=20_000, n_polys=400),
    "zipf": lambda: syn.zipf_join(seed=13, n_points=40_000, n_polys=1_500),
    "lattice": _lattice,
}


def _sorted(l, r, d=None):
    o = np.lexsort((r, l))
    return (l[o], r[o]) if d is None else (l[o], r[o], d[o])


@pytest.mark.parametrize("name", sorted(WORKLOADS))
@pytest.mark.parametrize("learned", [False, True])
def test_dwithin_matches_oracle(ctx, vsabi, oracle, name, learned):
    rng = np.random.default_rng(5)
    w = _with_outside_points(WORKLOADS[name](), rng)
    index, pts, keep = _device(vsabi, ctx, w, learned=learned)
    P = _oracle_polys(oracle, w)
    span = float(np.nanmax(w.polys.x) - np.nanmin(w.polys.x))
    for d in (0.0, 1e-3 * span, 0.02 * span, 0.5 * span, -1.0, np.nan):
        el, er, _ = oracle.dwithin_join(w.px, w.py, None, P, d)
        gl, gr, st = index.dwithin(pts, distance=d)
        np.testing.assert_array_equal(gl.cpu().numpy(), el, err_msg=f"{name} d={d}")
        np.testing.assert_array_equal(gr.cpu().numpy(), er, err_msg=f"{name} d={d}")
    # per-point distances with zeros, negatives and NaNs
    n = len(w.px)
    dp = rng.uniform(0, 0.05 * span, n)
    dp[rng.random(n) < 0.1] = 0.0
    dp[rng.random(n) < 0.05] = -1.0
    dp[rng.random(n) < 0.05] = np.nan
    el, er, _ = oracle.dwithin_join(w.px, w.py, None, P, point_distance=dp)
    import torch

    gl, gr, _ = index.dwithin(pts, point_distance=torch.from_numpy(dp).cuda())
    np.testing.assert_array_equal(gl.cpu().numpy(), el)
    np.testing.assert_array_equal(gr.cpu().numpy(), er)
    # per-polygon distances
    m = len(w.polys.geom_off) - 1
    dg = rng.uniform(0, 0.05 * span, m)
    dg[rng.random(m) < 0.1] = np.nan
    el, er, _ = oracle.dwithin_join(w.px, w.py, None, P, geom_distance=dg)
    gl, gr, _ = index.dwithin(pts, geom_distance=torch.from_numpy(dg).cuda())
    np.testing.assert_array_equal(gl.cpu().numpy(), el)
    np.testing.assert_array_equal(gr.cpu().numpy(), er)


@pytest.mark.parametrize("name", sorted(WORKLOADS))
@pytest.mark.parametrize("learned", [False, True])
def test_nearest_matches_oracle(ctx, vsabi, oracle, name, learned):
    rng = np.random.default_rng(6)
    w = _with_outside_points(WORKLOADS[name](), rng)
    index, pts, keep = _device(vsabi, ctx, w, learned=learned)
    P = _oracle_polys(oracle, w)
    span = float(np.nanmax(w.polys.x) - np.nanmin(w.polys.x))
    for md in (np.inf, 0.0, 0.01 * span, 0.3 * span):
        el, er, ed = oracle.nearest_join(w.px, w.py, None, P, md)
        gl, gr, gd, st = index.nearest(pts, max_distance=md)
        gl, gr, gd = gl.cpu().numpy(), gr.cpu().numpy(), gd.cpu().numpy()
        np.testing.assert_array_equal(gl, el, err_msg=f"{name} max_distance={md}")
        np.testing.assert_array_equal(gr, er, err_msg=f"{name} max_distance={md}")
        np.testing.assert_array_equal(gd.view(np.int64), ed.view(np.int64), err_msg=f"{name} max_distance={md}")
    if name == "lattice":
        # points on shared edges and vertices tie between 2 and 4 squares
        counts = np.bincount(el, minlength=len(w.px))
        assert counts.max() == 4 and (counts == 2).any()


def test_distance_joins_nulls_and_capacity(ctx, vsabi, oracle):
    rng = np.random.default_rng(7)
    w = syn.degenerate_join(seed=14, n_points=8_000, n_polys=300)
    pvalid = rng.random(len(w.px)) > 0.1
    gvalid = rng.random(len(w.polys.geom_off) - 1) > 0.2
    index, pts, keep = _device(vsabi, ctx, w, pvalid=pvalid, gvalid=gvalid)
    P = _oracle_polys(oracle, w, gvalid.astype(np.uint8))
    el, er, _ = oracle.dwithin_join(w.px, w.py, pvalid.astype(np.uint8), P, 3.0)
    gl, gr, _ = index.dwithin(pts, distance=3.0)
    np.testing.assert_array_equal(gl.cpu().numpy(), el)
    np.testing.assert_array_equal(gr.cpu().numpy(), er)
    el, er, ed = oracle.nearest_join(w.px, w.py, pvalid.astype(np.uint8), P)
    gl, gr, gd, _ = index.nearest(pts)
    np.testing.assert_array_equal(gl.cpu().numpy(), el)
    np.testing.assert_array_equal(gr.cpu().numpy(), er)
    np.testing.assert_array_equal(gd.cpu().numpy(), ed)
    # a pair buffer that is too small reports the exact size
    import torch

    small = torch.empty(10, dtype=torch.int32, device="cuda")
    with pytest.raises(vsabi.CapacityError) as e:
        index.nearest_into(pts, small, small.clone())
    assert e.value.required == len(el)
    with pytest.raises(vsabi.CapacityError) as e:
        index.dwithin_into(pts, small, small.clone(), distance=3.0)
    assert e.value.required > 10


def test_distance_joins_empty_sides(ctx, vsabi):
    import torch

    w = syn.star_join(seed=15, n_points=100, n_polys=10)
    index, pts, keep = _device(vsabi, ctx, w)
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    none = vsabi.make_points(e, e.clone())
    l, r, _ = index.dwithin(none, distance=1.0)
    assert l.numel() == 0
    l, r, d, _ = index.nearest(none)
    assert l.numel() == 0
    # every polygon null: no pairs
    index2, pts2, keep2 = _device(vsabi, ctx, w, gvalid=np.zeros(10, bool))
    assert index2.dwithin(pts2, distance=1e9)[0].numel() == 0
    assert index2.nearest(pts2)[0].numel() == 0


@pytest.mark.parametrize("name", ["star", "degenerate", "lattice"])
def test_distance_aligned_matches_oracle(ctx, vsabi, oracle, name):
    import torch

    w = WORKLOADS[name]()
    p = w.polys
    m = len(p.geom_off) - 1
    rng = np.random.default_rng(9)
    idx = rng.choice(len(w.px), m, replace=len(w.px) < m)
    px, py = w.px[idx].copy(), w.py[idx].copy()
    px[::17] = np.nan
    pvalid = (np.arange(m) % 13 != 0).astype(np.uint8)
    gvalid = (np.arange(m) % 11 != 0).astype(np.uint8)
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k))).cuda()
         for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    gv = torch.from_numpy(gvalid).cuda()
    P = vsabi.make_polygons(t["x"], t["y"], t["ring_off"], t["part_off"], t["geom_off"], gv)
    dx, dy, dv = (torch.from_numpy(a).cuda() for a in (px, py, pvalid))
    pts = vsabi.make_points(dx, dy, dv)
    dist = torch.empty(m, dtype=torch.float64, device="cuda")
    env = torch.empty(m, dtype=torch.float64, device="cuda")
    vsabi.distance_aligned(ctx, pts, P, dist, env)
    ed, ee = oracle.distance_aligned(px, py, pvalid, _oracle_polys(oracle, w, gvalid))
    np.testing.assert_array_equal(dist.cpu().numpy().view(np.int64), ed.view(np.int64))
    np.testing.assert_array_equal(env.cpu().numpy().view(np.int64), ee.view(np.int64))
    assert np.isnan(ed[::13]).all() and (ed[np.isfinite(ed)] >= 0).all()


@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_nearest_polygons_matches_oracle(ctx, vsabi, oracle, name):
    """The reverse query (nearest points of every polygon) against the oracle."""
    import torch

    rng = np.random.default_rng(10)
    w = _with_outside_points(WORKLOADS[name](), rng)
    n = len(w.px)
    m = len(w.polys.geom_off) - 1
    pvalid = (rng.random(n) > 0.05).astype(np.uint8)
    gvalid = (rng.random(m) > 0.05).astype(np.uint8)
    dx, dy, dv = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (w.px, w.py, pvalid))
    pidx = vsabi.point_index(ctx, dx, dy, dv)
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(w.polys, k))).cuda()
         for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    gv = torch.from_numpy(gvalid).cuda()
    P = vsabi.make_polygons(t["x"], t["y"], t["ring_off"], t["part_off"], t["geom_off"], gv)
    OP = _oracle_polys(oracle, w, gvalid)
    span = float(np.nanmax(w.polys.x) - np.nanmin(w.polys.x))
    for md in (np.inf, 0.0, 0.01 * span):
        el, er, ed = oracle.nearest_polygons_join(w.px, w.py, pvalid, OP, md)
        gl, gr, gd, _ = vsabi.nearest_polygons(ctx, pidx, P, max_distance=md)
        np.testing.assert_array_equal(gl.cpu().numpy(), el, err_msg=f"{name} max_distance={md}")
        np.testing.assert_array_equal(gr.cpu().numpy(), er, err_msg=f"{name} max_distance={md}")
        np.testing.assert_array_equal(gd.cpu().numpy().view(np.int64), ed.view(np.int64))
