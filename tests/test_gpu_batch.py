"""Batched joins (vs_batch_plan_create / vs_batch_run): every job's pairs equal
that job joined alone (vs_join) and the oracle, with and without the CUDA
graph, across launch shapes, predicates, null/NaN points and empty jobs."""
import numpy as np
import pytest

from _helpers import PRED_CODES, oracle_polys, to_dev, upload_points, upload_polys

pytestmark = pytest.mark.gpu


def _jobs(seed=7, n_jobs=12):
    from vibespatial_b200.testing import synthetic as syn

    return syn.batched_jobs(seed=seed, n_jobs=n_jobs, pts_range=(500, 60_000), poly_range=(3, 3000))


class _Batch:
    def __init__(self, abi, ctx, jobs, pvalid=None, options=None, empty_index_jobs=(), learned=False):
        self.jobs = jobs
        self.px = np.concatenate([w.px for w in jobs])
        self.py = np.concatenate([w.py for w in jobs])
        self.pvalid = pvalid
        self.job_start = np.concatenate([[0], np.cumsum([w.n_points for w in jobs])]).astype(np.int64)
        self.pts, self._pbufs = upload_points(abi, self.px, self.py, pvalid)
        self.indexes, self._keep = [], []
        for j, w in enumerate(jobs):
            P, bufs = upload_polys(abi, w.polys)
            if j in empty_index_jobs:  # every polygon row null
                bufs["valid"] = to_dev(np.zeros(len(w.polys.geom_off) - 1, np.uint8))
                P.d_valid = bufs["valid"].data_ptr()
            self._keep.append(bufs)
            self.indexes.append(abi.DeviceIndex(ctx, P, learned=learned))
        if learned:
            options = dict(options or {}, method=abi.METHOD_LEARNED)
        self.plan = abi.BatchPlan(ctx, self.indexes, self.pts, self.job_start, options=options)

    def split(self, left, right):
        """Pairs per job, local point rows, sorted by (left, right)."""
        job = np.searchsorted(self.job_start, left, side="right") - 1
        out = []
        for j in range(len(self.jobs)):
            m = job == j
            l, r = left[m] - self.job_start[j], right[m]
            o = np.lexsort((r, l))
            out.append((l[o], r[o]))
        return out


def _run(b, predicate, use_graph=True):
    left, right, stats = b.plan.run(PRED_CODES[predicate], use_graph=use_graph)
    return left.cpu().numpy().astype(np.int64), right.cpu().numpy().astype(np.int64), stats


@pytest.fixture(scope="module")
def batch(vsabi, ctx):
    return _Batch(vsabi, ctx, _jobs())


@pytest.mark.parametrize("predicate", ["within", "intersects", "touches", None])
def test_batch_matches_single_jobs_and_oracle(batch, vsabi, ctx, oracle, predicate):
    left, right, stats = _run(batch, predicate)
    assert len(left) == len(set(zip(left.tolist(), right.tolist())))  # no duplicates
    per_job = batch.split(left, right)
    for j, w in enumerate(batch.jobs):
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), predicate)
        np.testing.assert_array_equal(per_job[j][0], el)
        np.testing.assert_array_equal(per_job[j][1], er)
        # the same job through the single-join entry point
        sl = slice(batch.job_start[j], batch.job_start[j + 1])
        pts, _k = upload_points(vsabi, w.px, w.py)
        gl, gr, _ = batch.indexes[j].join(pts, PRED_CODES[predicate], vsabi.METHOD_RTREE, sort=True)
        np.testing.assert_array_equal(gl.cpu().numpy(), el)
        np.testing.assert_array_equal(gr.cpu().numpy(), er)
        assert sl.stop - sl.start == w.n_points
    assert stats["kernel_ms"] > 0


def test_graph_replay_and_direct_launch_agree(batch):
    a = _run(batch, "within", use_graph=True)
    b = _run(batch, "within", use_graph=True)  # replay of the captured graph
    c = _run(batch, "within", use_graph=False)
    sa, sb, sc = (batch.split(x[0], x[1]) for x in (a, b, c))
    for ja, jb, jc in zip(sa, sb, sc):
        np.testing.assert_array_equal(ja[0], jb[0])
        np.testing.assert_array_equal(ja[1], jb[1])
        np.testing.assert_array_equal(ja[0], jc[0])
        np.testing.assert_array_equal(ja[1], jc[1])


def test_graph_recaptures_when_buffers_change(batch, vsabi):
    import torch

    n_ref, _ = batch.plan.run_into(PRED_CODES["within"], *[torch.empty(1 << 20, dtype=torch.int32,
                                                                         device="cuda") for _ in range(2)])
    l2 = torch.full((n_ref + 7,), -1, dtype=torch.int32, device="cuda")
    r2 = torch.full((n_ref + 7,), -1, dtype=torch.int32, device="cuda")
    n2, _ = batch.plan.run_into(PRED_CODES["within"], l2, r2)
    assert n2 == n_ref
    assert int((l2[:n2] >= 0).sum()) == n2 and int((l2[n2:] == -1).sum()) == 7


def test_batch_capacity_error_reports_required(batch, vsabi):
    import torch

    left, right, _ = _run(batch, "intersects")
    small = [torch.empty(10, dtype=torch.int32, device="cuda") for _ in range(2)]
    with pytest.raises(vsabi.CapacityError) as ei:
        batch.plan.run_into(PRED_CODES["intersects"], *small)
    assert ei.value.required == len(left)


@pytest.mark.parametrize("options", [
    {"blocks_per_sm": 1, "packets_per_grab": 1, "sort_levels": 4},
    {"blocks_per_sm": 8, "packets_per_grab": 16, "sort_levels": 14},
    {"blocks_per_sm": 3, "packets_per_grab": 7, "sort_levels": 1},
])
def test_batch_launch_shapes_do_not_change_pairs(vsabi, ctx, oracle, options):
    jobs = _jobs(seed=11, n_jobs=5)
    b = _Batch(vsabi, ctx, jobs, options=options)
    left, right, _ = _run(b, "within")
    for j, (l, r) in enumerate(b.split(left, right)):
        w = jobs[j]
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "within")
        np.testing.assert_array_equal(l, el)
        np.testing.assert_array_equal(r, er)


def test_batch_null_nan_points_and_empty_jobs(vsabi, ctx, oracle):
    from vibespatial_b200.testing import synthetic as syn

    jobs = _jobs(seed=3, n_jobs=6)
    # a job with no points, and one whose polygons are all null
    jobs.insert(2, syn.star_join(seed=99, n_points=0, n_polys=20))
    n = sum(w.n_points for w in jobs)
    rng = np.random.default_rng(0)
    pvalid = (rng.random(n) > 0.1).astype(np.uint8)
    for w in jobs:
        if w.n_points:
            w.px[:: 97] = np.nan
    b = _Batch(vsabi, ctx, jobs, pvalid=pvalid, empty_index_jobs=(4,))
    left, right, _ = _run(b, "intersects")
    for j, (l, r) in enumerate(b.split(left, right)):
        w = jobs[j]
        if j == 4:
            assert len(l) == 0
            continue
        pv = pvalid[b.job_start[j]:b.job_start[j + 1]]
        el, er = oracle.join(w.px, w.py, pv, oracle_polys(oracle, w.polys), "intersects")
        np.testing.assert_array_equal(l, el)
        np.testing.assert_array_equal(r, er)


def test_batch_rejects_bad_arguments(vsabi, ctx, batch):
    with pytest.raises(ValueError):
        vsabi.BatchPlan(ctx, batch.indexes, batch.pts, batch.job_start[:-1])
    bad = batch.job_start.copy()
    bad[-1] += 1
    with pytest.raises(ValueError):
        vsabi.BatchPlan(ctx, batch.indexes, batch.pts, bad)
    bad = batch.job_start.copy()
    bad[2], bad[3] = bad[3], bad[2]
    with pytest.raises(ValueError):
        vsabi.BatchPlan(ctx, batch.indexes, batch.pts, bad)


def test_autotuned_options_round_trip(vsabi, ctx, batch, tmp_path):
    import torch

    from vibespatial_b200 import autotune as at

    left = torch.empty(1 << 20, dtype=torch.int32, device="cuda")
    right = torch.empty(1 << 20, dtype=torch.int32, device="cuda")
    n_polys = sum(len(w.polys.geom_off) - 1 for w in batch.jobs)
    path = tmp_path / "tune.json"
    opts = at.tuned_options(ctx, batch.indexes, batch.pts, batch.job_start, PRED_CODES["within"], n_polys,
                            left=left, right=right, passes=1, path=path)
    assert set(opts) == set(at.DEFAULTS)
    assert at.tuned_options(ctx, batch.indexes, batch.pts, batch.job_start, PRED_CODES["within"], n_polys,
                            left=left, right=right, path=path) == opts  # cache hit
    plan = vsabi.BatchPlan(ctx, batch.indexes, batch.pts, batch.job_start, options=opts)
    l1, r1, _ = plan.run(PRED_CODES["within"])
    l0, r0, _ = _run(batch, "within")
    a = batch.split(l1.cpu().numpy().astype(np.int64), r1.cpu().numpy().astype(np.int64))
    b = batch.split(l0, r0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x[0], y[0])
        np.testing.assert_array_equal(x[1], y[1])


# ---- learned method: the same batches through the learned cell indexes ----

@pytest.fixture(scope="module")
def lbatch(vsabi, ctx):
    return _Batch(vsabi, ctx, _jobs(), learned=True)


@pytest.mark.parametrize("predicate", ["within", "intersects", "touches", None])
@pytest.mark.parametrize("use_graph", [True, False])
def test_learned_batch_matches_oracle(lbatch, oracle, predicate, use_graph):
    left, right, _ = _run(lbatch, predicate, use_graph=use_graph)
    assert len(left) == len(set(zip(left.tolist(), right.tolist())))
    for j, (l, r) in enumerate(lbatch.split(left, right)):
        w = lbatch.jobs[j]
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), predicate)
        np.testing.assert_array_equal(l, el)
        np.testing.assert_array_equal(r, er)


@pytest.mark.parametrize("options", [
    {"learned_map_blocks_per_sm": 1, "learned_refine_blocks_per_sm": 1, "learned_grab": 32},
    {"learned_map_blocks_per_sm": 3, "learned_refine_blocks_per_sm": 2, "learned_grab": 100, "learned_map_packets": 2},
    {"learned_refine_blocks_per_sm": 5, "learned_map_packets": 2},
    {"learned_grab": 4096, "learned_flags": 4},
    {"learned_refine_blocks_per_sm": 8, "learned_flags": 8},
])
def test_learned_batch_launch_shapes_do_not_change_pairs(vsabi, ctx, oracle, options):
    """Learned batch plans give the oracle's pairs whatever their launch shape (the autotuner's search space)
    and with either ablation switch, graph-replayed and launched directly."""
    jobs = _jobs(seed=12, n_jobs=5)
    b = _Batch(vsabi, ctx, jobs, options=options, learned=True)
    for use_graph in (True, False):
        left, right, _ = _run(b, "intersects", use_graph=use_graph)
        for j, (l, r) in enumerate(b.split(left, right)):
            w = jobs[j]
            el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "intersects")
            np.testing.assert_array_equal(l, el)
            np.testing.assert_array_equal(r, er)


def test_learned_autotune_round_trip(vsabi, ctx, lbatch, tmp_path):
    """The autotuner searches the learned pipeline's launch shape, caches it, and the tuned plan gives the
    default plan's pairs."""
    import torch

    from vibespatial_b200 import autotune as at

    left = torch.empty(1 << 20, dtype=torch.int32, device="cuda")
    right = torch.empty(1 << 20, dtype=torch.int32, device="cuda")
    n_polys = sum(len(w.polys.geom_off) - 1 for w in lbatch.jobs)
    path = tmp_path / "tune.json"
    opts, src = at.tuned_options(ctx, lbatch.indexes, lbatch.pts, lbatch.job_start, PRED_CODES["within"], n_polys,
                                 left=left, right=right, passes=1, path=path, method=vsabi.METHOD_LEARNED,
                                 with_source=True)
    assert src == "searched" and set(opts) == set(at.LEARNED_DEFAULTS)
    again, src2 = at.tuned_options(ctx, lbatch.indexes, lbatch.pts, lbatch.job_start, PRED_CODES["within"],
                                   n_polys, left=left, right=right, path=path, method=vsabi.METHOD_LEARNED,
                                   with_source=True)
    assert (again, src2) == (opts, "cache")
    plan = vsabi.BatchPlan(ctx, lbatch.indexes, lbatch.pts, lbatch.job_start,
                           options=dict(opts, method=vsabi.METHOD_LEARNED))
    l1, r1, _ = plan.run(PRED_CODES["within"])
    l0, r0, _ = _run(lbatch, "within")
    for x, y in zip(lbatch.split(l1.cpu().numpy().astype(np.int64), r1.cpu().numpy().astype(np.int64)),
                    lbatch.split(l0, r0)):
        np.testing.assert_array_equal(x[0], y[0])
        np.testing.assert_array_equal(x[1], y[1])


def test_learned_batch_rejects_bad_shapes(vsabi, ctx, lbatch):
    for bad in ({"learned_grab": -1}, {"learned_map_blocks_per_sm": 9}, {"learned_flags": 1},
                {"learned_map_packets": 3}):
        with pytest.raises(ValueError):
            vsabi.BatchPlan(ctx, lbatch.indexes, lbatch.pts, lbatch.job_start,
                            options=dict(bad, method=vsabi.METHOD_LEARNED))


def test_learned_batch_single_job_equals_vs_join(vsabi, ctx):
    from vibespatial_b200.testing import synthetic as syn

    w = syn.zipf_join(seed=9, n_points=400_000, n_polys=8_000)
    b = _Batch(vsabi, ctx, [w], learned=True)
    left, right, _ = _run(b, "within")
    (l, r), = b.split(left, right)
    pts, _k = upload_points(vsabi, w.px, w.py)
    gl, gr, _ = b.indexes[0].join(pts, PRED_CODES["within"], vsabi.METHOD_LEARNED, sort=True)
    np.testing.assert_array_equal(l, gl.cpu().numpy())
    np.testing.assert_array_equal(r, gr.cpu().numpy())


def test_learned_batch_nulls_empty_jobs(vsabi, ctx, oracle):
    from vibespatial_b200.testing import synthetic as syn

    jobs = _jobs(seed=4, n_jobs=5)
    jobs.insert(1, syn.star_join(seed=98, n_points=0, n_polys=10))
    n = sum(w.n_points for w in jobs)
    pvalid = (np.random.default_rng(2).random(n) > 0.2).astype(np.uint8)
    b = _Batch(vsabi, ctx, jobs, pvalid=pvalid, empty_index_jobs=(3,), learned=True)
    left, right, _ = _run(b, "intersects")
    for j, (l, r) in enumerate(b.split(left, right)):
        if j == 3:
            assert len(l) == 0
            continue
        w = jobs[j]
        pv = pvalid[b.job_start[j]:b.job_start[j + 1]]
        el, er = oracle.join(w.px, w.py, pv, oracle_polys(oracle, w.polys), "intersects")
        np.testing.assert_array_equal(l, el)
        np.testing.assert_array_equal(r, er)


def test_learned_batch_needs_learned_indexes(vsabi, ctx, batch):
    with pytest.raises(ValueError):
        vsabi.BatchPlan(ctx, batch.indexes, batch.pts, batch.job_start, options={"method": vsabi.METHOD_LEARNED})


@pytest.mark.parametrize("learned", [False, True])
def test_batch_deferred_buffer_grows(vsabi, ctx, oracle, learned):
    """On-edge points defer more pairs than the plan's first buffer holds: the plan grows it and reruns."""
    from vibespatial_b200.testing import synthetic as syn

    w = syn.degenerate_join(seed=6, n_points=1_000_000, n_polys=10_000)
    b = _Batch(vsabi, ctx, [w], learned=learned)
    for use_graph in (True, True, False):
        left, right, stats = _run(b, "intersects", use_graph=use_graph)
        (l, r), = b.split(left, right)
        el, er = oracle.join(w.px, w.py, None, oracle_polys(oracle, w.polys), "intersects")
        np.testing.assert_array_equal(l, el)
        np.testing.assert_array_equal(r, er)
        assert stats["exact_fallbacks"] > 0
