"""Join export on the device (vs_join_export) against the host export
(sjoin._join_indexers on numpy arrays, the reference's _adjust_join_indexers
steps): identical output rows and source pairs for every ``how``, with and
without attribute codes."""
import importlib

import numpy as np
import pytest

vs_sjoin = importlib.import_module("vibespatial_b200.sjoin")

pytestmark = pytest.mark.gpu


def _pairs(rng, n_left, n_right, n_pairs):
    l = rng.integers(0, n_left, n_pairs)
    r = rng.integers(0, n_right, n_pairs)
    u = np.unique(l.astype(np.int64) * n_right + r)
    return (u // n_right).astype(np.int32), (u % n_right).astype(np.int32)


def _codes(rng, n, k, miss=0.1):
    c = rng.integers(0, k, n).astype(np.int64)
    c[rng.random(n) < miss] = -1
    return c


@pytest.mark.parametrize("how", ["inner", "left", "right", "outer"])
@pytest.mark.parametrize("with_codes", [False, True])
# sizes: (left rows, right rows, pairs drawn); the export writes tiles of 2048
# driving rows, so the cases cross tile edges (4096, 2049 rows) and give
# single driving rows thousands of pairs (3 right rows, 20k pairs)
@pytest.mark.parametrize("sizes", [(1000, 300, 5000), (50_000, 20_000, 400_000), (7, 5, 0), (0, 9, 0), (5, 0, 0),
                                   (3000, 3, 20_000), (4096, 2049, 30_000), (2049, 1, 2049)])
def test_export_matches_host(ctx, vsabi, how, with_codes, sizes):
    import torch

    n_left, n_right, n_pairs = sizes
    rng = np.random.default_rng(n_left + 7 * n_right + n_pairs)
    l, r = _pairs(rng, max(n_left, 1), max(n_right, 1), n_pairs) if n_left and n_right else (
        np.zeros(0, np.int32), np.zeros(0, np.int32))
    codes = (_codes(rng, n_left, 5), _codes(rng, n_right, 5)) if with_codes else None
    el, er, es = vs_sjoin._join_indexers(l, r, n_left, n_right, how, codes)
    dl = torch.from_numpy(l).cuda()
    dr = torch.from_numpy(r).cuda()
    lc = None if codes is None else torch.from_numpy(codes[0]).cuda()
    rc = None if codes is None else torch.from_numpy(codes[1]).cuda()
    gl, gr, gs = vsabi.join_export(ctx, dl, dr, n_left, n_right, how, lc, rc)
    np.testing.assert_array_equal(gl.cpu().numpy(), el)
    np.testing.assert_array_equal(gr.cpu().numpy(), er)
    np.testing.assert_array_equal(gs.cpu().numpy(), es)


def test_export_rejects_out_of_range_pairs(ctx, vsabi):
    import torch

    l = torch.tensor([0, 1, 5], dtype=torch.int32, device="cuda")
    r = torch.tensor([0, 0, 0], dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        vsabi.join_export(ctx, l, r, 3, 2, "left")
    with pytest.raises(ValueError):
        vsabi.join_export(ctx, l[:2], r[:2], 3, 2, "left", torch.zeros(3, dtype=torch.int64, device="cuda"))
    # with codes on both sides the attribute filter checks the ranges
    codes_l = torch.zeros(3, dtype=torch.int64, device="cuda")
    codes_r = torch.zeros(2, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError):
        vsabi.join_export(ctx, l, r, 3, 2, "left", codes_l, codes_r)
    with pytest.raises(ValueError):
        vsabi.join_export(ctx, l[:2], r[:2] - 1, 3, 2, "inner", codes_l, codes_r)
