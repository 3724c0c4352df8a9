"""Multi-GPU layout of the join: query points sharded, polygon index replicated.

Each point's pairs depend only on the read-only polygon side, so the join
partitions into independent units: rank r joins the r-th contiguous slice of
the points against its own replica of the index, with no collective on the
data path (weak scaling).  The only collective is optional bookkeeping after
the join: an all-gather of the per-rank pair counts, so every rank knows
where its pairs start in the concatenated result.  One process per GPU,
``torch.distributed`` for the plumbing (NCCL on GPUs, gloo on CPU).
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


def sharded_join(points, polygons, predicate="within", *, method="learned", pairs_fn=None, gather_counts=True):
    """This rank's pairs (global point rows) and, optionally, every rank's pair count.

    ``points`` / ``polygons`` are GeometryArrays (the same on every rank);
    ``pairs_fn(points, polygons, predicate)`` defaults to the CUDA join.
    Returns (left, right, counts) where counts is None unless gathered.
    """
    dist, rank, world = _dist()
    start, stop = shard_range(len(points), rank, world)
    local = points.take(np.arange(start, stop))
    if pairs_fn is None:
        from ._device import join_pairs

        left, right = join_pairs(local, polygons, predicate, method=method)
    else:
        left, right = pairs_fn(local, polygons, predicate)
    left = np.asarray(left, dtype=np.int64) + start
    right = np.asarray(right, dtype=np.int64)
    counts = None
    if gather_counts and dist is not None:
        import torch

        backend = dist.get_backend()
        device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        mine = torch.tensor([len(left)], dtype=torch.int64, device=device)
        allc = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
        dist.all_gather(allc, mine)
        counts = np.array([int(c.item()) for c in allc], dtype=np.int64)
    elif gather_counts:
        counts = np.array([len(left)], dtype=np.int64)
    return left, right, counts
