"""Row reductions of a join's pairs on the device (vs_row_counts, vs_row_sums,
vs_select_rows, vs_pairs_member) against numpy: counts and masked counts,
per-row sums bit for bit with numpy's bincount(weights=...), semijoin and
antijoin row sets, pair membership, and the argument errors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n_pairs, n_rows", [(0, 5), (1, 1), (1000, 7), (300_001, 50_000), (2_000_000, 3)])
def test_row_counts_and_masks(vsabi, ctx, n_pairs, n_rows):
    rng = np.random.default_rng(n_pairs + n_rows)
    rows = rng.integers(0, n_rows, n_pairs).astype(np.int32)
    rows_sorted = np.sort(rows)
    mask = rng.random(n_pairs) < 0.3
    for r in (rows, rows_sorted):
        got = vsabi.row_counts(ctx, _dev(r), n_rows).cpu().numpy()
        np.testing.assert_array_equal(got, np.bincount(r, minlength=n_rows))
        got = vsabi.row_counts(ctx, _dev(r), n_rows, mask=_dev(mask)).cpu().numpy()
        np.testing.assert_array_equal(got, np.bincount(r[mask], minlength=n_rows))


def test_row_sums_match_numpy_bit_for_bit(vsabi, ctx):
    rng = np.random.default_rng(3)
    n_rows, n_vals = 20_000, 1_000
    rows = np.sort(rng.integers(0, n_rows, 400_000)).astype(np.int32)
    rows[:5000] = 7  # one long run
    rows = np.sort(rows)
    cols = rng.integers(0, n_vals, len(rows)).astype(np.int32)
    vals = rng.standard_normal(n_vals) * 10.0 ** rng.integers(-8, 8, n_vals)
    got = vsabi.row_sums(ctx, _dev(rows), _dev(cols), _dev(vals), n_rows).cpu().numpy()
    exp = np.bincount(rows, weights=vals[cols], minlength=n_rows)
    np.testing.assert_array_equal(got.view(np.int64), exp.view(np.int64))
    with pytest.raises(ValueError, match="sorted by row"):
        vsabi.row_sums(ctx, _dev(rows[::-1].copy()), _dev(cols), _dev(vals), n_rows)
    bad = cols.copy()
    bad[10] = n_vals
    with pytest.raises(ValueError, match="column"):
        vsabi.row_sums(ctx, _dev(rows), _dev(bad), _dev(vals), n_rows)


def test_select_rows_semijoin_and_antijoin(vsabi, ctx):
    rng = np.random.default_rng(4)
    for n in (1, 31, 100_003):
        counts = rng.integers(0, 3, n).astype(np.int64)
        got = vsabi.select_rows(ctx, _dev(counts), True).cpu().numpy()
        np.testing.assert_array_equal(got, np.flatnonzero(counts > 0))
        got = vsabi.select_rows(ctx, _dev(counts), False).cpu().numpy()
        np.testing.assert_array_equal(got, np.flatnonzero(counts == 0))


def test_pairs_member(vsabi, ctx):
    rng = np.random.default_rng(5)
    n_left, n_right = 5_000, 900
    a = np.unique(rng.integers(0, n_left * n_right, 60_000))
    b = np.unique(np.concatenate([a[::3], rng.integers(0, n_left * n_right, 30_000)]))
    al, ar = (a // n_right).astype(np.int32), (a % n_right).astype(np.int32)
    bl, br = (b // n_right).astype(np.int32), (b % n_right).astype(np.int32)
    perm = rng.permutation(len(al))  # a in any order; b sorted by (left, right)
    got = vsabi.pairs_member(ctx, _dev(al[perm]), _dev(ar[perm]), _dev(bl), _dev(br), n_left).cpu().numpy()
    np.testing.assert_array_equal(got, np.isin(a[perm], b))
    with pytest.raises(ValueError, match="sorted"):
        vsabi.pairs_member(ctx, _dev(al), _dev(ar), _dev(bl[::-1].copy()), _dev(br[::-1].copy()), n_left)


def test_row_range_errors(vsabi, ctx):
    rows = np.array([0, 1, 5], np.int32)
    with pytest.raises(ValueError, match="outside"):
        vsabi.row_counts(ctx, _dev(rows), 5)
    with pytest.raises(ValueError, match="outside"):
        vsabi.row_counts(ctx, _dev(np.array([-1], np.int32)), 5)
