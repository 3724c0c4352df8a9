"""Multi-GPU layout of the joins: the query side sharded, the index replicated.

Each query row's pairs depend only on the read-only indexed side, so every
join here partitions into independent units: rank r joins its shard of the
query rows against its own replica of the index, with no collective on the
data path.  The query rows are the points for the predicate join, dwithin
and nearest (polygons indexed), and the polygons for the reverse nearest
join (points indexed).

Shards are either contiguous slices of the rows (``shard="contiguous"``) or
ranges of the points' Hilbert keys (``shard="hilbert"``): the rows sorted by
the level-16 Hilbert key of the point on the frame of all points, cut into
``world`` runs of equal size, so each rank holds a spatially compact set of
points and touches only the part of the index around it.

After the join, the per-rank pair counts are all-gathered (so every rank
knows where its pairs start in the concatenated result) and, with
``assemble=True``, every rank sends its pairs to rank 0, which receives them
in rank order (point-to-point sends sized by the gathered counts) and
returns the whole pair set sorted by (left, right).  One process per GPU,
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


def hilbert_keys_np(x, y, frame=None, level: int = 16) -> np.ndarray:
    """Level-``level`` Hilbert keys (uint32, level <= 16) of points on ``frame``
    (minx, miny, maxx, maxy; default: the finite points' bounds).  The same
    curve as the device keys (quadrant recursion, MSB first, swap / complement
    state).  NaN points get the all-ones key, so they sort last."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    ok = np.isfinite(x) & np.isfinite(y)
    if frame is None:
        frame = (x[ok].min(), y[ok].min(), x[ok].max(), y[ok].max()) if ok.any() else (0.0, 0.0, 1.0, 1.0)
    x0, y0, x1, y1 = (float(v) for v in frame)
    side = (1 << level) - 1
    with np.errstate(invalid="ignore"):
        gx = np.clip(np.nan_to_num((x - x0) / max(x1 - x0, 1e-300) * side), 0, side).astype(np.uint32)
        gy = np.clip(np.nan_to_num((y - y0) / max(y1 - y0, 1e-300) * side), 0, side).astype(np.uint32)
    key = np.zeros(len(x), np.uint32)
    sw = np.zeros(len(x), bool)
    inv = np.zeros(len(x), np.uint32)
    for lv in range(level - 1, -1, -1):
        bx = (gx >> np.uint32(lv)) & np.uint32(1)
        by = (gy >> np.uint32(lv)) & np.uint32(1)
        rx = np.where(sw, by, bx) ^ inv
        ry = np.where(sw, bx, by) ^ inv
        key = (key << np.uint32(2)) | ((np.uint32(3) * rx) ^ ry)
        turn = ry == 0
        inv = np.where(turn & (rx == 1), inv ^ np.uint32(1), inv)
        sw = np.where(turn, ~sw, sw)
    key[~ok] = np.uint32(0xFFFFFFFF)
    return key


def hilbert_shard_rows(x, y, rank: int, world: int, frame=None) -> np.ndarray:
    """Rows of ``rank``'s Hilbert-range shard: the rows ordered by their
    points' Hilbert keys (ties by row) and cut into ``world`` runs whose sizes
    differ by at most one.  Every row lands in exactly one shard; a shard's
    rows come back in key order."""
    start, stop = shard_range(len(x), rank, world)
    order = np.argsort(hilbert_keys_np(x, y, frame), kind="stable")
    return order[start:stop].astype(np.int64)


def shard_rows(query, rank: int, world: int, shard: str = "contiguous") -> np.ndarray:
    """Global rows of ``rank``'s shard of a GeometryArray of query rows."""
    if shard == "contiguous":
        start, stop = shard_range(len(query), rank, world)
        return np.arange(start, stop, dtype=np.int64)
    if shard == "hilbert":
        if not query.is_points():
            raise ValueError("Hilbert-range shards need a point array as the query side")
        x, y, valid = query.point_buffers()
        x = np.where(np.asarray(valid, bool), x, np.nan)
        return hilbert_shard_rows(x, y, rank, world)
    raise ValueError(f"shard must be 'contiguous' or 'hilbert', got {shard!r}")


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


def assemble_pairs(counts, *arrays, dst: int = 0):
    """Gather every rank's pair arrays on rank ``dst``, in rank order.

    ``counts`` are the all-gathered per-rank pair counts; ``arrays`` this
    rank's (left, right[, distances]) host arrays, of the same dtypes on every
    rank.  Each rank with pairs sends its arrays to ``dst`` (point-to-point,
    sized by the counts, so no rank waits on a message that is not sent).
    Returns the concatenated arrays on ``dst`` and None elsewhere; without a
    process group, the arrays themselves."""
    dist, rank, world = _dist()
    arrays = [np.ascontiguousarray(a) for a in arrays]
    if dist is None:
        return tuple(arrays)
    import torch

    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    if rank != dst:
        if counts[rank] > 0:
            for a in arrays:
                dist.send(torch.from_numpy(a).to(device), dst=dst)
        return None
    parts = [[] for _ in arrays]
    for r in range(world):
        if r == dst:
            for k, a in enumerate(arrays):
                parts[k].append(a)
            continue
        n = int(counts[r])
        if n == 0:
            continue
        for k, a in enumerate(arrays):
            buf = torch.empty(n, dtype=torch.from_numpy(a[:0]).dtype, device=device)
            dist.recv(buf, src=r)
            parts[k].append(buf.cpu().numpy())
    return tuple(np.concatenate(p) if p else a[:0] for p, a in zip(parts, arrays))


def _sharded(query, run, gather_counts, shard="contiguous", assemble=False):
    """Run ``run(local query rows, rows)`` on this rank's shard (``rows`` = the
    shard's global rows); the first returned array holds local query rows,
    mapped here to global rows.  With ``assemble``, rank 0 returns every
    rank's pairs sorted by (left, right) and the other ranks return None in
    place of their arrays."""
    _, rank, world = _dist()
    rows = shard_rows(query, rank, world, shard)
    out = list(run(query.take(rows), rows))
    out[0] = rows[np.asarray(out[0], dtype=np.int64)] if len(rows) else np.asarray(out[0], dtype=np.int64)
    out[1] = np.asarray(out[1], dtype=np.int64)
    counts = _gather_counts(len(out[0])) if (gather_counts or assemble) else None
    if assemble:
        got = assemble_pairs(counts, *out)
        if got is None:
            out = [None] * len(out)
        else:
            out = list(got)
            order = np.lexsort((out[1], out[0]))
            out = [a[order] for a in out]
    return (*out, counts)


def sharded_join(points, polygons, predicate="within", *, method="learned", pairs_fn=None, gather_counts=True,
                 shard="contiguous", assemble=False):
    """This rank's pairs (global point rows) and, optionally, every rank's pair count.

    ``points`` / ``polygons`` are GeometryArrays (the same on every rank);
    ``pairs_fn(points, polygons, predicate)`` defaults to the CUDA join.
    ``shard`` picks contiguous slices or Hilbert ranges of the points;
    ``assemble`` gathers the whole sorted pair set on rank 0 (None elsewhere).
    Returns (left, right, counts) where counts is None unless gathered.
    """
    def run(local, rows):
        if pairs_fn is not None:
            return pairs_fn(local, polygons, predicate)
        from ._device import join_pairs

        return join_pairs(local, polygons, predicate, method=method)

    return _sharded(points, run, gather_counts, shard, assemble)


def sharded_dwithin(points, polygons, *, distance=None, point_distance=None, geom_distance=None, method="learned",
                    pairs_fn=None, gather_counts=True, shard="contiguous", assemble=False):
    """dwithin over sharded points: (left, right, counts) as :func:`sharded_join`.
    A per-point distance array is sliced with the points; per-polygon or scalar
    distances are the same on every rank.  ``pairs_fn(points, polygons, **dist)``
    defaults to the CUDA join."""
    def run(local, rows):
        dist = {"distance": distance, "geom_distance": geom_distance}
        if point_distance is not None:
            dist["point_distance"] = np.asarray(point_distance, np.float64)[rows]
        dist = {k: v for k, v in dist.items() if v is not None}
        if pairs_fn is not None:
            return pairs_fn(local, polygons, **dist)
        from ._device import dwithin_pairs

        return dwithin_pairs(local, polygons, method=method, **dist)

    return _sharded(points, run, gather_counts, shard, assemble)


def sharded_nearest(points, polygons, *, max_distance=None, method="learned", pairs_fn=None, gather_counts=True,
                    shard="contiguous", assemble=False):
    """Nearest polygons of sharded points: (left, right, distances, counts).
    ``pairs_fn(points, polygons, max_distance=...)`` defaults to the CUDA join."""
    def run(local, rows):
        if pairs_fn is not None:
            return pairs_fn(local, polygons, max_distance=max_distance)
        from ._device import nearest_pairs

        return nearest_pairs(local, polygons, max_distance=max_distance, method=method)

    return _sharded(points, run, gather_counts, shard, assemble)


def sharded_nearest_polygons(polygons, points, *, max_distance=None, pairs_fn=None, gather_counts=True,
                             assemble=False):
    """Nearest points of sharded polygons (the points' index replicated):
    (polygon rows, point rows, distances, counts).  ``pairs_fn(polygons,
    points, max_distance=...)`` defaults to the CUDA join."""
    def run(local, rows):
        if pairs_fn is not None:
            return pairs_fn(local, points, max_distance=max_distance)
        from ._device import nearest_polygon_pairs

        return nearest_polygon_pairs(local, points, max_distance=max_distance)

    return _sharded(polygons, run, gather_counts, "contiguous", assemble)
