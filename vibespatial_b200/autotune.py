"""Autotuner for the batched join's launch shape.

The R-tree batch (``vs_batch_run`` with ``VS_METHOD_RTREE``) has three shape
parameters: join-kernel blocks per SM, 32-point packets a warp takes per grab
of the work counter, and the Hilbert levels the points of a job are sorted by
(more levels: coherent packets but more radix passes).  The learned batch
(``VS_METHOD_LEARNED``) has four of its own: map-pass blocks per SM, the
32-point packets a map warp looks up together (1 or 2), refine blocks per SM
(4 or fewer run the 64-register refine build, 5 the 48-register one), and the
grouped points a refine warp takes per grab of its work counter.  The best values depend on the device and on the batch's shape
(job count, points per job, polygons per job), so they are searched by timing
the real kernels and cached on disk per (device, shape class, predicate,
method).

The search is coordinate descent over a small grid: starting from the
defaults, each parameter in turn is swept with the others held, and the sweep
repeats until a pass improves nothing (at most ``passes`` times).  A candidate
is timed as the median device time of a few graph replays after a warm-up.
The reference tunes nothing at run time (its launch shapes are constants in
src/vibespatial/spatial/spatial_index_device.py:110-150); this module is the
project's own.
"""
from __future__ import annotations

import json
import math
import os
import tempfile
import threading
from pathlib import Path
from typing import Callable

DEFAULTS = {"blocks_per_sm": 4, "packets_per_grab": 4, "sort_levels": 8}
SPACE = {
    "blocks_per_sm": (2, 3, 4, 6, 8),
    "packets_per_grab": (1, 2, 4, 8, 16),
    "sort_levels": (6, 8, 10, 12),
}
LEARNED_DEFAULTS = {"learned_map_blocks_per_sm": 8, "learned_map_packets": 1, "learned_refine_blocks_per_sm": 4,
                    "learned_grab": 32}
LEARNED_SPACE = {
    "learned_map_blocks_per_sm": (2, 4, 6, 8),
    "learned_map_packets": (1, 2),
    "learned_refine_blocks_per_sm": (2, 3, 4, 5),
    "learned_grab": (32, 64, 128, 256),
}
METHOD_RTREE, METHOD_LEARNED = 0, 1


def space_for(method: int) -> tuple[dict, dict]:
    """(defaults, search space) of a batch method's launch shape."""
    return (LEARNED_DEFAULTS, LEARNED_SPACE) if int(method) == METHOD_LEARNED else (DEFAULTS, SPACE)
CACHE_ENV = "VIBESPATIAL_B200_AUTOTUNE_CACHE"
_lock = threading.Lock()


def cache_path() -> Path:
    p = os.environ.get(CACHE_ENV)
    if p:
        return Path(p)
    return Path(os.environ.get("XDG_CACHE_HOME", Path.home() / ".cache")) / "vibespatial_b200" / "autotune.json"


def shape_class(n_jobs: int, n_points: int, n_polygons: int) -> str:
    """Bucket of a batch shape: log2 buckets of jobs, points per job, polygons per job."""
    n_jobs = max(int(n_jobs), 1)

    def lg(v):
        return int(math.floor(math.log2(max(float(v), 1.0))))

    return f"j{lg(n_jobs)}-p{lg(n_points / n_jobs)}-g{lg(n_polygons / n_jobs)}"


def cache_key(device_name: str, sm_count: int, shape: str, predicate: int, method: int = METHOD_RTREE) -> str:
    key = f"{device_name}|sm{int(sm_count)}|{shape}|pred{int(predicate)}"
    return key if int(method) == METHOD_RTREE else f"{key}|learned"


def load_cache(path: Path | None = None) -> dict:
    p = path or cache_path()
    try:
        with open(p) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def store(key: str, options: dict, ms: float, path: Path | None = None) -> None:
    """Merge one entry into the cache file (atomic replace)."""
    p = path or cache_path()
    with _lock:
        data = load_cache(p)
        data[key] = {"options": {k: int(v) for k, v in options.items()}, "ms": float(ms)}
        p.parent.mkdir(parents=True, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=str(p.parent), prefix=".autotune-", suffix=".json")
        with os.fdopen(fd, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, p)


def lookup(key: str, path: Path | None = None, method: int = METHOD_RTREE) -> dict | None:
    ent = load_cache(path).get(key)
    if not ent or not isinstance(ent.get("options"), dict):
        return None
    defaults, _ = space_for(method)
    opts = dict(defaults)
    opts.update({k: int(v) for k, v in ent["options"].items() if k in defaults})
    return opts


def search(measure: Callable[[dict], float], space: dict | None = None, start: dict | None = None,
           passes: int = 2) -> tuple[dict, float, list]:
    """Coordinate descent: returns (best options, best ms, [(options, ms), ...] tried).

    ``measure(options) -> ms`` times one candidate; each distinct candidate is
    measured once.
    """
    space = space or SPACE
    best = dict(start or DEFAULTS)
    seen: dict[tuple, float] = {}
    tried = []

    def cost(o):
        k = tuple(sorted(o.items()))
        if k not in seen:
            seen[k] = float(measure(dict(o)))
            tried.append((dict(o), seen[k]))
        return seen[k]

    best_ms = cost(best)
    for _ in range(max(int(passes), 1)):
        improved = False
        for name, values in space.items():
            for v in values:
                if v == best.get(name):
                    continue
                cand = dict(best)
                cand[name] = v
                ms = cost(cand)
                if ms < best_ms:
                    best, best_ms, improved = cand, ms, True
        if not improved:
            break
    return best, best_ms, tried


def device_identity(device: int = 0) -> tuple[str, int]:
    import torch

    prop = torch.cuda.get_device_properties(device)
    return prop.name, int(prop.multi_processor_count)


def time_plan(plan, predicate: int, left, right, *, warmup: int = 2, reps: int = 5) -> float:
    """Median device time (ms) of graph replays of ``plan``."""
    for _ in range(warmup):
        plan.run_into(predicate, left, right, use_graph=True)
    ms = sorted(plan.run_into(predicate, left, right, use_graph=True)[1]["kernel_ms"] for _ in range(reps))
    return ms[len(ms) // 2]


def tuned_options(ctx, indexes, pts, job_start, predicate: int, n_polygons: int, *, left, right,
                  use_cache: bool = True, passes: int = 2, path: Path | None = None,
                  method: int = METHOD_RTREE, with_source: bool = False):
    """Launch shape for this batch and method: from the cache, else searched
    and stored.  With ``with_source``, returns (options, "cache"|"searched").

    ``left`` / ``right`` are pair buffers large enough for the batch (the
    search runs the real join into them).  The options exclude ``method``.
    """
    from ._abi import BatchPlan

    defaults, space = space_for(method)
    name, sms = device_identity(ctx.device)
    key = cache_key(name, sms, shape_class(len(indexes), int(pts.n), n_polygons), predicate, method)
    if use_cache:
        hit = lookup(key, path, method)
        if hit is not None:
            return (hit, "cache") if with_source else hit

    def measure(opts):
        plan = BatchPlan(ctx, indexes, pts, job_start, options=dict(opts, method=int(method)))
        try:
            return time_plan(plan, predicate, left, right)
        finally:
            plan.close()

    best, ms, _ = search(measure, space=space, start=defaults, passes=passes)
    store(key, best, ms, path)
    return (best, "searched") if with_source else best
