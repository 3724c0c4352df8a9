"""Row-flow carriers of the index queries: pairs, row sets and per-row values.

The reference's spatial index hands its native callers three private carriers
instead of exported numpy pairs: ``NativeRelation`` (relation pairs, query rows
on the left, src/vibespatial/api/_native_relation.py:381), ``NativeRowSet`` /
``NativeDeviceSelection`` (row positions of one side,
src/vibespatial/api/_native_rowset.py:882) and ``NativeExpression`` (one value
per row, src/vibespatial/api/_native_expression.py:321).  These are the same
three shapes over this package's join output: the arrays are the CUDA tensors
the join returned (or numpy arrays when a test substitutes the pair source),
and every reduction between them (counts, semijoins, complements) runs where
the arrays live.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np


def _is_numpy(a) -> bool:
    return isinstance(a, np.ndarray)


def _size(a) -> int:
    return int(a.shape[0]) if _is_numpy(a) else int(a.numel())


def _ctx(t):
    from . import _abi

    return _abi, _abi.default_context(t.device.index if t.device.index is not None else 0)


def _counts(rows, n: int, mask=None):
    """Occurrences of 0..n-1 in ``rows`` (int64, same device as ``rows``), over
    the pairs where ``mask`` is set when given; device arrays are counted by
    the library's row-count kernel (vs_row_counts)."""
    if _is_numpy(rows):
        r = rows.astype(np.int64) if mask is None else rows[np.asarray(mask, bool)].astype(np.int64)
        return np.bincount(r, minlength=n)[:n].astype(np.int64) if len(r) else np.zeros(n, np.int64)
    abi, ctx = _ctx(rows)
    return abi.row_counts(ctx, rows, n, mask)


def _matched_rows(counts, matched: bool = True):
    """Ascending rows whose count is > 0 (``matched``) or == 0: the
    semijoin / antijoin row sets (vs_select_rows on the device)."""
    if _is_numpy(counts):
        return np.flatnonzero(counts > 0 if matched else counts == 0).astype(np.int64)
    abi, ctx = _ctx(counts)
    return abi.select_rows(ctx, counts, matched)


def _nonzero(flags):
    if _is_numpy(flags):
        return np.flatnonzero(flags).astype(np.int64)
    return flags.nonzero().flatten()


def _to_numpy(a) -> np.ndarray:
    return a if _is_numpy(a) else a.cpu().numpy()


@dataclass
class Relation:
    """Relation pairs: ``left_indices[k]`` (query row) relates to
    ``right_indices[k]`` (indexed row); ``distances`` per pair for nearest."""

    left_indices: Any
    right_indices: Any
    predicate: str | None = None
    distances: Any | None = None
    left_row_count: int | None = None
    right_row_count: int | None = None
    sorted_by_left: bool = False

    def __len__(self) -> int:
        return _size(self.left_indices)

    @property
    def is_device(self) -> bool:
        return not _is_numpy(self.left_indices)

    def left_match_count_expression(self) -> "Expression":
        """Matches per query row."""
        return Expression("relation.left_match_count", _counts(self.left_indices, int(self.left_row_count)),
                          source_row_count=int(self.left_row_count), dtype="int64")

    def right_match_count_expression(self) -> "Expression":
        """Matches per indexed row."""
        return Expression("relation.right_match_count", _counts(self.right_indices, int(self.right_row_count)),
                          source_row_count=int(self.right_row_count), dtype="int64")

    def left_semijoin_rowset(self) -> "RowSet":
        """Query rows with at least one match, ascending."""
        c = self.left_match_count_expression().values
        return RowSet(_matched_rows(c, True), source_row_count=int(self.left_row_count), unique=True)

    def left_antijoin_rowset(self) -> "RowSet":
        """Query rows without any match, ascending."""
        c = self.left_match_count_expression().values
        return RowSet(_matched_rows(c, False), source_row_count=int(self.left_row_count), unique=True)

    def right_semijoin_rowset(self) -> "RowSet":
        """Indexed rows with at least one match, ascending."""
        c = self.right_match_count_expression().values
        return RowSet(_matched_rows(c, True), source_row_count=int(self.right_row_count), unique=True)

    def to_numpy(self) -> np.ndarray:
        """The (2, K) intp pairs of sindex.query."""
        return np.vstack([_to_numpy(self.left_indices).astype(np.intp),
                          _to_numpy(self.right_indices).astype(np.intp)]) if len(self) else np.empty((2, 0), np.intp)


@dataclass
class RowSet:
    """Ascending row positions of one side (``source_row_count`` rows)."""

    positions: Any
    source_row_count: int | None = None
    ordered: bool = True
    unique: bool = True

    def __len__(self) -> int:
        return _size(self.positions)

    @property
    def is_device(self) -> bool:
        return not _is_numpy(self.positions)

    def mask(self):
        """Boolean flags over the source rows."""
        n = int(self.source_row_count)
        if _is_numpy(self.positions):
            m = np.zeros(n, bool)
            m[self.positions] = True
            return m
        import torch

        m = torch.zeros(n, dtype=torch.bool, device=self.positions.device)
        if self.positions.numel():
            m[self.positions.long()] = True
        return m

    def complement(self) -> "RowSet":
        """The source rows not in this set, ascending."""
        return RowSet(_nonzero(~self.mask()), source_row_count=self.source_row_count)

    def to_numpy(self) -> np.ndarray:
        return _to_numpy(self.positions).astype(np.intp)


@dataclass
class Expression:
    """One value per source row (``values`` has ``source_row_count`` rows)."""

    operation: str
    values: Any
    source_row_count: int | None = None
    dtype: str | None = None

    def __post_init__(self) -> None:
        if self.source_row_count is not None and len(self) != int(self.source_row_count):
            raise ValueError("Expression source_row_count must match expression length")

    def __len__(self) -> int:
        return _size(self.values)

    @property
    def is_device(self) -> bool:
        return not _is_numpy(self.values)

    def to_numpy(self) -> np.ndarray:
        return _to_numpy(self.values)

    def compare_scalar_selection(self, op: str, value) -> RowSet:
        """Rows whose value compares true against ``value`` (``op`` one of
        ``>``, ``>=``, ``<``, ``<=``, ``==``, ``!=``)."""
        import operator

        ops = {">": operator.gt, ">=": operator.ge, "<": operator.lt, "<=": operator.le, "==": operator.eq,
               "!=": operator.ne}
        if op not in ops:
            raise ValueError(f"unsupported comparison {op!r}")
        return RowSet(_nonzero(ops[op](self.values, value)), source_row_count=self.source_row_count)
