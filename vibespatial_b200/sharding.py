"""Multi-GPU layout of the joins: the query side sharded, the index replicated.

Each query row's pairs depend only on the read-only indexed side, so every
join here partitions into independent units: rank r joins the r-th
contiguous slice of the query rows against its own replica of the index,
with no collective on the data path (weak scaling).  The query rows are the
points for the predicate join, dwithin and nearest (polygons indexed), and
the polygons for the reverse nearest join (points indexed).  The only
collective is optional bookkeeping after the join: an all-gather of the
per-rank pair counts, so every rank knows where its pairs start in the
concatenated result.  One process per GPU, ``torch.distributed`` for the
plumbing (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced [start, stop) slice of n items for ``rank``."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world size {world}")
    base, extra = divmod(int(n), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist, dist.get_rank(), dist.get_world_size()
    return None, 0, 1


def _gather_counts(n_local: int):
    """Every rank's pair count (the all-gather), or this rank's alone."""
    dist, _, world = _dist()
    if dist is None:
        return np.array([n_local], dtype=np.int64)
    import torch

    backend = dist.get_backend()
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    mine = torch.tensor([n_local], dtype=torch.int64, device=device)
    allc = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(allc, mine)
    return np.array([int(c.item()) for c in allc], dtype=np.int64)


def _sharded(query, run, gather_counts):
    """Run ``run(local query rows, start)`` on this rank's slice; the first
    returned array holds local query rows, shifted here to global rows."""
    _, rank, world = _dist()
    start, stop = shard_range(len(query), rank, world)
    out = list(run(query.take(np.arange(start, stop)), start))
    out[0] = np.asarray(out[0], dtype=np.int64) + start
    out[1] = np.asarray(out[1], dtype=np.int64)
    counts = _gather_counts(len(out[0])) if gather_counts else None
    return (*out, counts)


def sharded_join(points, polygons, predicate="within", *, method="learned", pairs_fn=None, gather_counts=True):
    """This rank's pairs (global point rows) and, optionally, every rank's pair count.

    ``points`` / ``polygons`` are GeometryArrays (the same on every rank);
    ``pairs_fn(points, polygons, predicate)`` defaults to the CUDA join.
    Returns (left, right, counts) where counts is None unless gathered.
    """
    def run(local, start):
        if pairs_fn is not None:
            return pairs_fn(local, polygons, predicate)
        from ._device import join_pairs

        return join_pairs(local, polygons, predicate, method=method)

    return _sharded(points, run, gather_counts)


def sharded_dwithin(points, polygons, *, distance=None, point_distance=None, geom_distance=None, method="learned",
                    pairs_fn=None, gather_counts=True):
    """dwithin over sharded points: (left, right, counts) as :func:`sharded_join`.
    A per-point distance array is sliced with the points; per-polygon or scalar
    distances are the same on every rank.  ``pairs_fn(points, polygons, **dist)``
    defaults to the CUDA join."""
    def run(local, start):
        dist = {"distance": distance, "geom_distance": geom_distance}
        if point_distance is not None:
            dist["point_distance"] = np.asarray(point_distance, np.float64)[start:start + len(local)]
        dist = {k: v for k, v in dist.items() if v is not None}
        if pairs_fn is not None:
            return pairs_fn(local, polygons, **dist)
        from ._device import dwithin_pairs

        return dwithin_pairs(local, polygons, method=method, **dist)

    return _sharded(points, run, gather_counts)


def sharded_nearest(points, polygons, *, max_distance=None, method="learned", pairs_fn=None, gather_counts=True):
    """Nearest polygons of sharded points: (left, right, distances, counts).
    ``pairs_fn(points, polygons, max_distance=...)`` defaults to the CUDA join."""
    def run(local, start):
        if pairs_fn is not None:
            return pairs_fn(local, polygons, max_distance=max_distance)
        from ._device import nearest_pairs

        return nearest_pairs(local, polygons, max_distance=max_distance, method=method)

    return _sharded(points, run, gather_counts)


def sharded_nearest_polygons(polygons, points, *, max_distance=None, pairs_fn=None, gather_counts=True):
    """Nearest points of sharded polygons (the points' index replicated):
    (polygon rows, point rows, distances, counts).  ``pairs_fn(polygons,
    points, max_distance=...)`` defaults to the CUDA join."""
    def run(local, start):
        if pairs_fn is not None:
            return pairs_fn(local, points, max_distance=max_distance)
        from ._device import nearest_polygon_pairs

        return nearest_polygon_pairs(local, points, max_distance=max_distance)

    return _sharded(polygons, run, gather_counts)
