"""Sharded join across ranks (gloo, world size 2, CPU): the union of the ranks'
pairs equals the single-process join, and the gathered counts locate them."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_shard_range_covers_everything_once():
    from vibespatial_b200.sharding import shard_range

    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_hilbert_keys_follow_the_device_curve():
    """The host keys that cut Hilbert-range shards are the device curve's keys (16 levels)."""
    from vibespatial_b200 import _abi
    from vibespatial_b200.sharding import hilbert_keys_np

    rng = np.random.default_rng(4)
    x = rng.uniform(-5, 5, 2000)
    y = rng.uniform(10, 30, 2000)
    frame = (-5.0, 10.0, 5.0, 30.0)
    keys = hilbert_keys_np(x, y, frame)
    side = (1 << 16) - 1
    gx = np.clip((x + 5.0) / 10.0 * side, 0, side).astype(np.uint32)
    gy = np.clip((y - 10.0) / 20.0 * side, 0, side).astype(np.uint32)
    exp = [_abi.hilbert_key_host(int(a) << 16, int(b) << 16, 16) for a, b in zip(gx, gy)]
    np.testing.assert_array_equal(keys, np.array(exp, np.uint32))
    x[::5] = np.nan
    assert (hilbert_keys_np(x, y, frame)[::5] == 0xFFFFFFFF).all()


def test_hilbert_shards_partition_rows_and_stay_compact():
    from vibespatial_b200.sharding import hilbert_shard_rows

    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1000, 100_003)
    y = rng.uniform(0, 1000, 100_003)
    x[::97] = np.nan  # empty points go to the last shard
    for world in (1, 2, 3, 4, 8):
        shards = [hilbert_shard_rows(x, y, r, world) for r in range(world)]
        allr = np.concatenate(shards)
        assert len(allr) == len(x) and len(np.unique(allr)) == len(x)
        sizes = [len(s) for s in shards]
        assert max(sizes) - min(sizes) <= 1
        if world == 4:  # a quarter of uniform points covers well under the whole frame's box
            for s in shards[:-1]:
                area = np.ptp(x[s]) * np.ptp(y[s])
                assert area < 0.6 * 1000 * 1000, area
    assert np.isnan(x[hilbert_shard_rows(x, y, 3, 4)[-1]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    import oracle as O
    from vibespatial_b200.geometry import GeometryArray
    from vibespatial_b200.sharding import sharded_join
    from vibespatial_b200.testing import synthetic as syn

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w = syn.star_join(seed=31, n_points=30_001, n_polys=300)
        points = GeometryArray.from_points(w.px, w.py)
        polys = GeometryArray.from_polygon_buffers(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off,
                                                   w.polys.geom_off)

        def pairs_fn(pts, pg, predicate):  # the CPU oracle stands in for the GPU join here
            px, py, pv = pts.point_buffers()
            pb = pg.polygon_buffers()
            return O.join(px, py, pv, O.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid),
                          predicate)

        left, right, counts = sharded_join(points, polys, "within", pairs_fn=pairs_fn)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), left=left, right=right, counts=counts)
        # Hilbert-range shards, pairs assembled on rank 0 (None elsewhere)
        al, ar, ac = sharded_join(points, polys, "within", pairs_fn=pairs_fn, shard="hilbert", assemble=True)
        if rank == 0:
            np.savez(os.path.join(out_dir, "assembled.npz"), left=al, right=ar, counts=ac)
        else:
            assert al is None and ar is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_join(tmp_path, oracle):
    import torch.multiprocessing as mp

    from vibespatial_b200.testing import synthetic as syn

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    counts = parts[0]["counts"]
    assert np.array_equal(counts, parts[1]["counts"])
    assert [len(p["left"]) for p in parts] == counts.tolist()
    left = np.concatenate([p["left"] for p in parts])
    right = np.concatenate([p["right"] for p in parts])
    w = syn.star_join(seed=31, n_points=30_001, n_polys=300)
    el, er = oracle.join(w.px, w.py, None, oracle.Polygons(w.polys.x, w.polys.y, w.polys.ring_off,
                                                          w.polys.part_off, w.polys.geom_off), "within")
    o = np.lexsort((right, left))
    np.testing.assert_array_equal(left[o], el)
    np.testing.assert_array_equal(right[o], er)
    # rank 0 holds the lower half of the points
    assert parts[0]["left"].max() < parts[1]["left"].min()
    # Hilbert-range shards assembled on rank 0: the single-process pair set, sorted
    a = np.load(tmp_path / "assembled.npz")
    np.testing.assert_array_equal(a["left"], el)
    np.testing.assert_array_equal(a["right"], er)
    assert a["counts"].sum() == len(el) and (a["counts"] > 0).all()


def _distance_worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    import oracle as O
    from vibespatial_b200.geometry import GeometryArray
    from vibespatial_b200.sharding import sharded_dwithin, sharded_nearest, sharded_nearest_polygons
    from vibespatial_b200.testing import synthetic as syn

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w = syn.star_join(seed=33, n_points=8_001, n_polys=201)
        points = GeometryArray.from_points(w.px, w.py)
        polys = GeometryArray.from_polygon_buffers(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off,
                                                   w.polys.geom_off)

        def oracle_args(pts, pg):  # the CPU oracle stands in for the GPU joins here
            px, py, pv = pts.point_buffers()
            pb = pg.polygon_buffers()
            return px, py, pv, O.Polygons(pb.x, pb.y, pb.ring_off, pb.part_off, pb.geom_off, pb.valid)

        def dwithin_fn(pts, pg, distance=0.0, point_distance=None, geom_distance=None):
            px, py, pv, P = oracle_args(pts, pg)
            l, r, _ = O.dwithin_join(px, py, pv, P, distance, point_distance=point_distance,
                                     geom_distance=geom_distance)
            return l, r

        def nearest_fn(pts, pg, max_distance=None):
            px, py, pv, P = oracle_args(pts, pg)
            return O.nearest_join(px, py, pv, P, float("inf") if max_distance is None else max_distance)

        def nearest_polygons_fn(pg, pts, max_distance=None):
            px, py, pv, P = oracle_args(pts, pg)
            return O.nearest_polygons_join(px, py, pv, P, float("inf") if max_distance is None else max_distance)

        per_point = np.linspace(0.0, 3.0, len(w.px))
        out = {}
        out["dw_l"], out["dw_r"], out["dw_c"] = sharded_dwithin(points, polys, point_distance=per_point,
                                                                pairs_fn=dwithin_fn)
        out["nn_l"], out["nn_r"], out["nn_d"], out["nn_c"] = sharded_nearest(points, polys, max_distance=25.0,
                                                                             pairs_fn=nearest_fn)
        out["np_l"], out["np_r"], out["np_d"], out["np_c"] = sharded_nearest_polygons(polys, points,
                                                                                     pairs_fn=nearest_polygons_fn)
        # distances travel with their pairs through the assembly
        hl, hr, hd, hc = sharded_nearest(points, polys, max_distance=25.0, pairs_fn=nearest_fn, shard="hilbert",
                                         assemble=True)
        if rank == 0:
            out["hn_l"], out["hn_r"], out["hn_d"] = hl, hr, hd
        dist.barrier()
        np.savez(os.path.join(out_dir, f"dist_rank{rank}.npz"), **out)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_distance_joins(tmp_path, oracle):
    """dwithin (per-point distances sliced with the points), nearest (points
    sharded) and reverse nearest (polygons sharded): the ranks' pairs
    together are the single-process result, the gathered counts locate them."""
    import torch.multiprocessing as mp

    from vibespatial_b200.testing import synthetic as syn

    world = 2
    mp.start_processes(_distance_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    parts = [np.load(tmp_path / f"dist_rank{r}.npz") for r in range(world)]
    w = syn.star_join(seed=33, n_points=8_001, n_polys=201)
    P = oracle.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    per_point = np.linspace(0.0, 3.0, len(w.px))
    expected = {
        "dw": oracle.dwithin_join(w.px, w.py, None, P, 0.0, point_distance=per_point)[:2],
        "nn": oracle.nearest_join(w.px, w.py, None, P, 25.0),
        "np": oracle.nearest_polygons_join(w.px, w.py, None, P),
    }
    for key, exp in expected.items():
        counts = parts[0][f"{key}_c"]
        assert np.array_equal(counts, parts[1][f"{key}_c"])
        assert [len(p[f"{key}_l"]) for p in parts] == counts.tolist()
        got = [np.concatenate([p[f"{key}_{c}"] for p in parts]) for c in ("l", "r", "d")[:len(exp)]]
        # the ranks hold consecutive slices of the query rows, each sorted: concatenated, they are sorted
        for g, e in zip(got, exp):
            np.testing.assert_array_equal(g, e)
        assert len(got[0]) > 0
    for g, e in zip((parts[0]["hn_l"], parts[0]["hn_r"], parts[0]["hn_d"]), expected["nn"]):
        np.testing.assert_array_equal(g, e)


@pytest.mark.gpu
def test_sharded_joins_one_rank_on_the_gpu(oracle):
    """Without a process group the sharded forms are the whole join on the
    CUDA path: same pairs and distances as the oracle."""
    from vibespatial_b200.geometry import GeometryArray
    from vibespatial_b200.sharding import sharded_dwithin, sharded_join, sharded_nearest, sharded_nearest_polygons
    from vibespatial_b200.testing import synthetic as syn

    w = syn.star_join(seed=35, n_points=20_000, n_polys=300)
    points = GeometryArray.from_points(w.px, w.py)
    polys = GeometryArray.from_polygon_buffers(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off,
                                               w.polys.geom_off)
    P = oracle.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    l, r, c = sharded_join(points, polys, "within")
    el, er = oracle.join(w.px, w.py, None, P, "within")
    np.testing.assert_array_equal(l, el)
    np.testing.assert_array_equal(r, er)
    assert c.tolist() == [len(el)]
    l, r, c = sharded_dwithin(points, polys, distance=1.5)
    el, er, _ = oracle.dwithin_join(w.px, w.py, None, P, 1.5)
    np.testing.assert_array_equal(l, el)
    np.testing.assert_array_equal(r, er)
    l, r, d, c = sharded_nearest(points, polys, max_distance=30.0)
    el, er, ed = oracle.nearest_join(w.px, w.py, None, P, 30.0)
    for g, e in ((l, el), (r, er), (d, ed)):
        np.testing.assert_array_equal(g, e)
    l, r, d, c = sharded_nearest_polygons(polys, points)
    el, er, ed = oracle.nearest_polygons_join(w.px, w.py, None, P)
    for g, e in ((l, el), (r, er), (d, ed)):
        np.testing.assert_array_equal(g, e)
