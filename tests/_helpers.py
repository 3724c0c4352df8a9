"""Shared test helpers: upload workloads, run the CUDA join, compare with the oracle."""
from __future__ import annotations

import numpy as np

PRED_CODES = {None: 0, "intersects": 1, "within": 2, "covered_by": 3, "touches": 4}


def oracle_polys(O, p):
    return O.Polygons(p.x, p.y, p.ring_off, p.part_off, p.geom_off, getattr(p, "valid", None))


def to_dev(a, dev="cuda"):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def upload_polys(abi, p):
    bufs = dict(x=to_dev(p.x), y=to_dev(p.y), ring_off=to_dev(p.ring_off), part_off=to_dev(p.part_off),
                geom_off=to_dev(p.geom_off))
    valid = getattr(p, "valid", None)
    bufs["valid"] = None if valid is None else to_dev(np.asarray(valid, np.uint8))
    return abi.make_polygons(bufs["x"], bufs["y"], bufs["ring_off"], bufs["part_off"], bufs["geom_off"],
                             bufs["valid"]), bufs


def upload_points(abi, px, py, pvalid=None):
    bufs = dict(x=to_dev(px), y=to_dev(py), valid=None if pvalid is None else to_dev(np.asarray(pvalid, np.uint8)))
    return abi.make_points(bufs["x"], bufs["y"], bufs["valid"]), bufs


def gpu_join(abi, ctx, px, py, polys, predicate="within", method=0, pvalid=None, learned=None, index=None):
    pts, keep1 = upload_points(abi, px, py, pvalid)
    if index is None:
        P, keep2 = upload_polys(abi, polys)
        index = abi.DeviceIndex(ctx, P, learned=(method == 1) if learned is None else learned)
    left, right, stats = index.join(pts, PRED_CODES[predicate], method, sort=True)
    return left.cpu().numpy(), right.cpu().numpy(), stats


def assert_same_pairs(got_l, got_r, exp_l, exp_r):
    assert len(got_l) == len(exp_l), f"pair count {len(got_l)} != oracle {len(exp_l)}"
    np.testing.assert_array_equal(got_l, exp_l)
    np.testing.assert_array_equal(got_r, exp_r)
