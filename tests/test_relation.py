"""Row-flow carriers (Relation, RowSet, Expression) over numpy arrays and
over CUDA tensors (the join's device output, reduced by the library's
row-reduction kernels), and SpatialIndex.query_pair_aggregate on device pairs."""
import numpy as np
import pytest
import torch

import vibespatial_b200 as vs
from vibespatial_b200 import query
from vibespatial_b200.relation import Expression, Relation, RowSet


KINDS = ["numpy", pytest.param("torch", marks=pytest.mark.gpu)]


@pytest.mark.parametrize("kind", KINDS)
def test_relation_reductions(kind):
    left = np.array([0, 0, 2, 2, 2, 5], np.int32)
    right = np.array([1, 3, 0, 1, 3, 3], np.int32)
    if kind == "torch":
        left, right = torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda()
    rel = Relation(left, right, predicate="intersects", left_row_count=7, right_row_count=4, sorted_by_left=True)
    assert len(rel) == 6 and rel.is_device == (kind == "torch")
    assert rel.left_match_count_expression().to_numpy().tolist() == [2, 0, 3, 0, 0, 1, 0]
    assert rel.right_match_count_expression().to_numpy().tolist() == [1, 2, 0, 3]
    semi = rel.left_semijoin_rowset()
    assert semi.to_numpy().tolist() == [0, 2, 5] and semi.source_row_count == 7
    assert semi.complement().to_numpy().tolist() == [1, 3, 4, 6]
    assert rel.left_antijoin_rowset().to_numpy().tolist() == [1, 3, 4, 6]
    assert rel.right_semijoin_rowset().to_numpy().tolist() == [0, 1, 3]
    assert rel.to_numpy().tolist() == [[0, 0, 2, 2, 2, 5], [1, 3, 0, 1, 3, 3]]


@pytest.mark.parametrize("kind", KINDS)
def test_empty_relation(kind):
    e = np.zeros(0, np.int32)
    left, right = (e, e.copy()) if kind == "numpy" else (torch.from_numpy(e).cuda(), torch.from_numpy(e.copy()).cuda())
    rel = Relation(left, right, left_row_count=3, right_row_count=2)
    assert len(rel) == 0 and rel.to_numpy().shape == (2, 0)
    assert rel.left_semijoin_rowset().to_numpy().tolist() == []
    assert rel.left_semijoin_rowset().complement().to_numpy().tolist() == [0, 1, 2]
    assert rel.right_match_count_expression().to_numpy().tolist() == [0, 0]


def test_expression_and_rowset_checks():
    with pytest.raises(ValueError, match="source_row_count"):
        Expression("x", np.zeros(3), source_row_count=4)
    ex = Expression("x", np.array([3, 0, 5]), source_row_count=3)
    assert ex.compare_scalar_selection(">=", 3).to_numpy().tolist() == [0, 2]
    assert ex.compare_scalar_selection("==", 0).to_numpy().tolist() == [1]
    rs = RowSet(torch.tensor([1, 4]), source_row_count=5)
    assert rs.mask().tolist() == [False, True, False, False, True]
    assert rs.complement().to_numpy().tolist() == [0, 2, 3]


@pytest.mark.gpu
def test_pair_aggregate_on_tensor_pairs(monkeypatch):
    """The device branch of query_pair_aggregate (vs_pairs_member and masked
    vs_row_counts on the pairs) gives the numpy branch's counts."""
    a_pairs = {"l": np.array([0, 1, 1, 3, 4, 4]), "r": np.array([0, 0, 1, 2, 0, 1])}
    b_pairs = {"l": np.array([0, 1, 1, 3]), "r": np.array([0, 0, 1, 3])}
    tree_a = vs.GeometryArray.from_shapes([vs.box(0, 0, 1, 1)] * 4)
    tree_b = vs.GeometryArray.from_shapes([vs.box(0, 0, 1, 1)] * 4)
    q = vs.GeoSeries([vs.Point(0.5, 0.5)] * 5)

    def fake_rows(as_tensor):
        def rows(self, arr, predicate, distance):
            p = a_pairs if self.geometry is tree_a else b_pairs
            l, r = p["l"].astype(np.int32), p["r"].astype(np.int32)
            return (torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()) if as_tensor else (l, r)
        return rows

    out = {}
    for as_tensor in (False, True):
        monkeypatch.setattr(query.SpatialIndex, "_pair_rows", fake_rows(as_tensor))
        out[as_tensor] = tree_a.sindex.query_pair_aggregate(tree_b.sindex, q, predicate="intersects")
    for df in out.values():
        assert df["left_count"].tolist() == [3, 2, 1, 0]
        assert df["right_count"].tolist() == [2, 1, 0, 1]
        assert df["shared_count"].tolist() == [2, 1, 0, 0]
