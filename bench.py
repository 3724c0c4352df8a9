"""Benchmark: query points/sec of the point-by-polygon join on B200.

Default workload (one JSON line on rank 0):
  zipf_join -- 50M FP64 points x 1M footprint polygons, cluster centres
  Zipf(s=1.1)-weighted over 1024 sites in [0,1000]^2 (the learned-index
  scale-up case), predicate 'within'.  A step = one join of all points
  against the resident polygon index (built once before timing, as an
  ``sindex`` is reused across queries).  Inputs (800 MB of points) exceed the
  126 MB L2, so no explicit flush is needed between steps.

Arms:
  --impl ours (default)  the CUDA path through the C-ABI (libvsjoin.so)
  --impl reference       the reference CPU path of this join, timed on the
                         host cores: the reference needs Shapely/GEOS, which
                         cannot be installed here, so the exact CPU oracle
                         (oracle/, C + OpenMP, kind "port") stands in for it.

Multi-GPU (torchrun, one rank per GPU): the join shards by query points; each
rank joins its own 50M-point batch against its replica of the index (weak
scaling, no collective on the data path).  Time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(name: str, rank: int = 0, scale: float = 1.0):
    from vibespatial_b200.testing import synthetic as syn

    if name == "zipf":
        return syn.zipf_join(seed=3 + 1000 * rank, n_points=int(50_000_000 * scale), n_polys=int(1_000_000 * scale))
    if name == "utm":
        return syn.utm_join(seed=1 + 1000 * rank, n_points=int(10_000_000 * scale), n_polys=int(100_000 * scale))
    if name == "star":
        return syn.star_join(seed=0 + 1000 * rank, n_points=int(100_000 * scale), n_polys=int(1_000 * scale))
    if name == "degenerate":
        return syn.degenerate_join(seed=5 + 1000 * rank, n_points=int(20_000_000 * scale),
                                   n_polys=int(200_000 * scale))
    raise ValueError(name)


PHASES = ("locate", "group", "refine", "exact")


def make_batched(rank: int = 0, scale: float = 1.0):
    from vibespatial_b200.testing import synthetic as syn

    return syn.batched_jobs(seed=2 + 1000 * rank, n_jobs=max(1, int(round(256 * scale))))


WORKLOAD_DESC = {
    "zipf": "zipf_join: 50M FP64 points x 1M footprints, Zipf(s=1.1) clusters over 1024 sites in [0,1000]^2",
    "utm": "utm_join: 10M FP64 points (64-component GMM) x 100k footprints, UTM-like frame",
    "star": "star_join: 100k points x 1k star polygons in [0,1000]^2",
    "degenerate": "degenerate_join: 20M points x 200k polygons with holes/multiparts, on-edge and 1-ulp points",
    "batched": "batched_jobs: 256 independent star joins, points logU[1k,2M] (69.6M total), polygons "
               "logU[10,50k] (1.38M total), one persistent launch replayed from a CUDA graph",
    "dwithin": "dwithin: zipf_join's 50M FP64 points x 1M footprints, pairs within distance 0.25 (1.7x the median "
               "footprint side)",
    "nearest": "nearest (sjoin_nearest, all ties, unbounded): zipf_join's 50M FP64 points x 1M footprints",
    "nearest_polygons": "nearest points of every polygon (sjoin_nearest with the polygons matched, all ties, "
                        "unbounded): zipf_join's 1M footprints x 50M points",
    "export": "join export: zipf_join's within pairs (50M points x 1M footprints) to how='left' row indexers "
              "(50M+ rows) after an on_attribute filter (codes row % 7 on both sides)",
    "wkb": "wkb ingest: the zipf_join inputs as little-endian 2D WKB columns (50M Points, 21 B each; 1M Polygons), "
           "decoded on the device into the join's columnar layout",
}


def algorithmic_bytes(w, n_pairs: int, n_points: int | None = None) -> int:
    """Bytes the join must move at least once: points, polygon SoA, pair output."""
    p = w.polys
    return int(16 * (w.n_points if n_points is None else n_points) + 16 * p.n_coords + 4 * (len(p.ring_off) + len(p.part_off) + len(p.geom_off))
               + 8 * n_pairs)


def plan_median_ms(plan, pred, left, right, n_expect, use_graph=True, reps=5, warm=2):
    """Median device time (CUDA events inside vs_batch_run) of a batch plan's join."""
    ms = []
    for k in range(warm + reps):
        n_k, st_k = plan.run_into(pred, left, right, use_graph=use_graph)
        assert n_k == n_expect, (n_k, n_expect)
        if k >= warm:
            ms.append(st_k["kernel_ms"])
    return float(np.median(ms))


def learned_ablations(_abi, ctx, indexes, pts, job_start, pred, left, right, n_pairs, base_opts, reps):
    """What each choice of the learned pipeline buys: the same batch plan with the RMI replaced by a binary
    search over every cell key, with FP64 ring walks instead of the FP32 stage, without the bulk-copy (TMA)
    staging of candidate records, without the interior-box shortcut, and launched directly instead of replayed
    from a CUDA graph (median device ms of each; same pairs)."""
    out = {}
    for name, extra, graph in (("graph_ms", {}, True), ("direct_launch_ms", {}, False),
                               ("rmi_replaced_by_bsearch_ms", {"learned_flags": _abi.JOIN_LEARNED_BSEARCH}, True),
                               ("fp64_walk_ms", {"learned_flags": _abi.JOIN_LEARNED_FP64_WALK}, True),
                               ("no_record_staging_ms", {"learned_flags": _abi.JOIN_LEARNED_NO_STAGE}, True),
                               ("no_interior_box_ms", {"learned_flags": _abi.JOIN_LEARNED_NO_INTERIOR}, True)):
        plan = _abi.BatchPlan(ctx, indexes, pts, job_start, options=dict(base_opts, **extra))
        out[name] = plan_median_ms(plan, pred, left, right, n_pairs, use_graph=graph, reps=reps)
        plan.close()
    return out


def workload_desc(args, name) -> str:
    """The workload's description; a --scale other than 1 is named in it (the sizes then differ from the text)."""
    scale = getattr(args, "scale", 1.0)
    return WORKLOAD_DESC[name] + (f" (scaled by {scale:g})" if scale != 1.0 else "")


def join_config(args, w) -> dict:
    """The workload's configuration, identical in both arms (arm-specific figures live outside it)."""
    return {"workload": workload_desc(args, args.workload), "predicate": args.predicate, "n_points_per_gpu": w.n_points,
            "n_polygons": len(w.polys), "l2": "inputs larger than L2 (126 MB); no flush"}


def batched_config(args, jobs) -> dict:
    return {"workload": workload_desc(args, "batched"), "predicate": args.predicate, "n_jobs": len(jobs),
            "n_points_per_gpu": int(sum(w.n_points for w in jobs)), "n_polygons": int(sum(len(w.polys) for w in jobs)),
            "l2": "inputs larger than L2 (126 MB); no flush"}


def every(stride, what) -> str:
    """'every point', 'every 2nd point', 'every 13th point'."""
    if stride <= 1:
        return f"every {what}"
    suffix = "th" if 10 <= stride % 100 <= 20 else {1: "st", 2: "nd", 3: "rd"}.get(stride % 10, "th")
    return f"every {stride}{suffix} {what}"


def shapely_importable() -> bool:
    """Whether Shapely (GEOS) imports on this host: the reference's own CPU path needs it."""
    try:
        import shapely  # noqa: F401
    except Exception:
        return False
    return True


def cpu_sample_rate(w, predicate: str, threads: int, target_s: float = 10.0):
    """Oracle (all host threads) on consecutive 2M-point chunks of the same
    points until ~target_s of work; (points/sec, points, seconds, pairs).
    When the chunks cover every point, `pairs` is the oracle's whole sorted
    (point row, polygon row) pair set (the checker of the GPU's pairs), else None."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    P = O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    chunk = min(w.n_points, 2_000_000)
    n, dt, start = 0, 0.0, 0
    ls, rs = [], []
    while dt < target_s and n < w.n_points:
        stop = min(start + chunk, w.n_points)
        t0 = time.perf_counter()
        l, r = O.join(w.px[start:stop], w.py[start:stop], None, P, predicate, threads)
        dt += time.perf_counter() - t0
        ls.append(l.astype(np.int64) + start)
        rs.append(r.astype(np.int64))
        n += stop - start
        start = stop
    pairs = (np.concatenate(ls), np.concatenate(rs)) if n == w.n_points and ls else None
    return n / dt, n, dt, pairs


def pair_mismatches(gl, gr, el, er) -> int:
    """Pairs in one set and not the other, plus repeated pairs (0 = bit-exact pair sets)."""
    a = (np.asarray(gl, np.int64) << 32) | np.asarray(gr, np.int64)
    b = (np.asarray(el, np.int64) << 32) | np.asarray(er, np.int64)
    ua, ub = np.unique(a), np.unique(b)
    return int(np.setxor1d(ua, ub, assume_unique=True).size + (len(a) - len(ua)) + (len(b) - len(ub)))


def cpu_sample_batched(jobs, predicate: str, threads: int, target_s: float = 10.0):
    """Oracle (all host threads) job after job until ~target_s of work; points/sec."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    n = 0
    dt = 0.0
    k = 0
    for w in jobs:
        P = O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
        t0 = time.perf_counter()
        O.join(w.px, w.py, None, P, predicate, threads)
        dt += time.perf_counter() - t0
        n += w.n_points
        k += 1
        if dt >= target_s:
            break
    return n / dt, n, dt, k


def run_reference_batched(args, world):
    jobs = make_batched(0, args.scale)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    # a bounded sample: every stride-th job (the sizes of the whole batch's
    # log-uniform spread), about --ref-sample points in all
    total = sum(w.n_points for w in jobs)
    stride = max(1, -(-total // max(1, args.ref_sample)))
    sample, n = [], 0
    for w in jobs[::stride]:
        sample.append((w, O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)))
        n += w.n_points

    def step():
        for w, P in sample:
            O.join(w.px, w.py, None, P, args.predicate, threads)

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * len(times) / tot
    line = {
        "impl": "reference", "metric": "query points/sec", "value": value, "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": batched_config(args, jobs),
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": "port",
                         "sample": f"{every(stride, 'job')} ({len(sample)} of {len(jobs)} jobs, {n} points), exact CPU "
                                   "oracle (C + OpenMP): Shapely/GEOS is not installable here",
                         "shapely_importable": shapely_importable()},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def make_wkb_columns(rank: int = 0, scale: float = 1.0):
    """The zipf_join inputs as WKB columns (Arrow binary layout: bytes, int64 offsets)."""
    from vibespatial_b200.testing import synthetic as syn

    w = make_workload("zipf", rank, scale)
    return w, [("points",) + syn.wkb_points(w.px, w.py), ("polygons",) + syn.wkb_polygons(w.polys)]


def wkb_algorithmic_bytes(n_rows: int, data_bytes: int, sz: dict) -> int:
    """Bytes a decode must move once: the WKB bytes and n + 1 int64 offsets in;
    tags, point x/y and geom_off per row, part_off, ring_off and x/y out."""
    return int(data_bytes + 8 * (n_rows + 1) + 17 * n_rows + 4 * (n_rows + 1) + 4 * (sz["n_parts"] + 1)
               + 4 * (sz["n_rings"] + 1) + 16 * sz["n_coords"])


def cpu_wkb_rate(cols, threads: int, target_s: float = 5.0):
    """CPU WKB decoder (oracle/wkb.c, all host threads) over whole columns until ~target_s; rows/sec."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    n, dt = 0, 0.0
    while dt < target_s:
        for _, data, off in cols:
            t0 = time.perf_counter()
            O.wkb_decode(data, off, None, threads)
            dt += time.perf_counter() - t0
            n += len(off) - 1
    return n / dt, n, dt


def run_reference_wkb(args, world):
    _, cols = make_wkb_columns(0, args.scale)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    rows = sum(len(off) - 1 for _, _, off in cols)
    for _ in range(args.warmup):
        for _, data, off in cols:
            O.wkb_decode(data, off, None, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for _, data, off in cols:
            O.wkb_decode(data, off, None, threads)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = rows * len(times) / tot
    line = {
        "impl": "reference", "metric": "WKB geometries decoded/sec", "value": value, "unit": "geometries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": workload_desc(args, "wkb"), "rows": rows},
        "cpu_baseline": {"value": value, "unit": "geometries/s", "cores": threads, "kind": "port",
                         "sample": "both whole columns each step, CPU WKB decoder (oracle/wkb.c, C + OpenMP) "
                                   "restating the reference's staged host decode"},
        "e2e": {"value": value, "unit": "geometries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_wkb(args, rank, world, local_rank):
    """WKB ingest: decode the join's two input columns on the device."""
    import torch

    from vibespatial_b200 import _abi

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
    w, cols = make_wkb_columns(rank, args.scale)
    ctx = _abi.Context(dev)
    stream = ctx.torch_stream
    d_cols = [(name, torch.from_numpy(d).to(dev), torch.from_numpy(o).to(dev)) for name, d, o in cols]
    rows = sum(len(o) - 1 for _, _, o in cols)
    data_bytes = sum(len(d) for _, d, _ in cols)
    # the decode reproduces the generator's columns exactly
    sz_p, out = _abi.wkb_decode(ctx, d_cols[0][1], d_cols[0][2])
    assert sz_p["n_points"] == w.n_points and sz_p["n_coords"] == 0
    assert torch.equal(out["px"].cpu(), torch.from_numpy(w.px)) and torch.equal(out["py"].cpu(), torch.from_numpy(w.py))
    sz_g, out = _abi.wkb_decode(ctx, d_cols[1][1], d_cols[1][2])
    for k in ("geom_off", "part_off", "ring_off", "x", "y"):
        assert np.array_equal(out[k].cpu().numpy(), getattr(w.polys, k)), k
    del out
    sizes = {"points": sz_p, "polygons": sz_g}

    def step(cs):
        return [_abi.wkb_decode(ctx, d, o)[0] for _, d, o in cs]

    for _ in range(args.warmup):
        step(d_cols)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = _abi.kernel_launches()
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            ev[k][0].record(stream)
            step(d_cols)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        launches = _abi.kernel_launches() - launches0
        # the size pass over the points column alone (one kernel + a 72-byte read of its totals)
        n_pts = len(cols[0][2]) - 1
        rows_out = {"tags": torch.empty(n_pts, dtype=torch.int8, device=dev),
                    "px": torch.empty(n_pts, dtype=torch.float64, device=dev),
                    "py": torch.empty(n_pts, dtype=torch.float64, device=dev),
                    "geom_off": torch.empty(n_pts + 1, dtype=torch.int32, device=dev)}
        size_ms = []
        for _ in range(max(3, args.steps)):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _abi.wkb_plan_sizes(ctx, d_cols[0][1], d_cols[0][2], None, rows_out)
            b.record(stream)
            torch.cuda.synchronize()
            size_ms.append(a.elapsed_time(b))
        # e2e: the columns from pinned host memory, copies inside the timed region
        h_cols = [(name, torch.from_numpy(d).pin_memory(), torch.from_numpy(o).pin_memory()) for name, d, o in cols]
        e2e_ms = []
        for k in range(max(3, args.steps) + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step([(name, d.to(dev, non_blocking=True), o.to(dev, non_blocking=True)) for name, d, o in h_cols])
            b.record(stream)
            torch.cuda.synchronize()
            if k:
                e2e_ms.append(a.elapsed_time(b))
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms, float(np.median(e2e_ms))], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        total_ms, e2e_med = float(t[0]), float(t[1])
    else:
        e2e_med = float(np.median(e2e_ms))
    value = world * rows * args.steps / (total_ms / 1e3)
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    smed = float(np.median(size_ms))
    B_size = int(len(cols[0][1]) + 8 * (n_pts + 1) + 17 * n_pts + 12 * n_pts)  # + the 3 per-row counts it writes
    B_alg = wkb_algorithmic_bytes(n_pts, len(cols[0][1]), sz_p)
    achieved = B_alg / (smed / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "traffic_wkb_points.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get("traffic_bytes_per_launch")
        except Exception:
            traffic = None
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        rate, n_s, dt = cpu_wkb_rate(cols, threads, min(args.cpu_seconds, 5.0))
        cpu = {"value": rate, "unit": "geometries/s", "cores": threads, "kind": "port",
               "sample": f"{n_s} rows of the same two columns ({dt:.1f} s), CPU WKB decoder (oracle/wkb.c, "
                         "C + OpenMP) restating the reference's staged host decode"}
    line = {
        "metric": "WKB geometries decoded/sec", "value": value, "unit": "geometries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": workload_desc(args, "wkb"), "rows": rows, "wkb_bytes": data_bytes,
                   "sizes": sizes, "parallelism": f"columns per GPU ({world} GPU(s)), independent",
                   "l2": "inputs (1.5 GB of WKB + offsets) larger than L2; no flush",
                   "api": "_abi.wkb_decode per column (plan with one host sync for the sizes, output "
                          "allocation, decode)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel": "wkb_size_kernel (points column)",
                     "kernel_ms": smed, "algorithmic_bytes_per_launch": B_alg, "bytes_moved_by_design": B_size},
        "cpu_baseline": cpu,
        "e2e": {"value": world * rows / (e2e_med / 1e3), "unit": "geometries/s",
                "h2d_bytes_per_step": int(sum(len(d) + 8 * len(o) for _, d, o in cols)),
                "d2h_bytes_per_step": 2 * 72},
        "gpu_launches": launches,
    }
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


DWITHIN_DISTANCE = 0.25


def cpu_distance_rate(w, kind: str, threads: int, target_s: float = 10.0):
    """CPU oracle of the distance join (grid index, all host threads) over
    consecutive 1M-point chunks until ~target_s; points/sec."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    P = O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    chunk = min(w.n_points, 1_000_000)
    n, dt, start = 0, 0.0, 0
    while dt < target_s and n < w.n_points:
        stop = min(start + chunk, w.n_points)
        t0 = time.perf_counter()
        if kind == "dwithin":
            O.dwithin_join(w.px[start:stop], w.py[start:stop], None, P, DWITHIN_DISTANCE, threads=threads)
        else:
            O.nearest_join(w.px[start:stop], w.py[start:stop], None, P, threads=threads)
        dt += time.perf_counter() - t0
        n += stop - start
        start = stop
    return n / dt, n, dt


def run_reference_distance(args, world):
    w = make_workload("zipf", 0, args.scale)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    P = O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    n = min(w.n_points, args.ref_sample // 4)

    def step():
        if args.workload == "dwithin":
            O.dwithin_join(w.px[:n], w.py[:n], None, P, DWITHIN_DISTANCE, threads=threads)
        else:
            O.nearest_join(w.px[:n], w.py[:n], None, P, threads=threads)

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * len(times) / tot
    line = {
        "impl": "reference", "metric": "query points/sec", "value": value, "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc(args, args.workload), "sample_points": n, "n_polygons": len(w.polys)},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": "port",
                         "sample": f"first {n} of {w.n_points} points vs all {len(w.polys)} polygons, CPU oracle "
                                   "(C + OpenMP, grid index, same distance arithmetic); Shapely/GEOS is not "
                                   "installable here"},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_distance(args, rank, world, local_rank):
    """dwithin / nearest over the zipf inputs through vs_join_dwithin / vs_join_nearest."""
    import torch

    from vibespatial_b200 import _abi

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
    w = make_workload("zipf", rank, args.scale)
    N = w.n_points
    ctx = _abi.Context(dev)
    stream = ctx.torch_stream
    pol = w.polys
    d_poly = {k: torch.from_numpy(np.ascontiguousarray(getattr(pol, k))).to(dev)
              for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    P = _abi.make_polygons(d_poly["x"], d_poly["y"], d_poly["ring_off"], d_poly["part_off"], d_poly["geom_off"])
    index = _abi.DeviceIndex(ctx, P, learned=False)
    dx = torch.from_numpy(w.px).to(dev)
    dy = torch.from_numpy(w.py).to(dev)
    pts = _abi.make_points(dx, dy)
    nearest = args.workload == "nearest"
    cap = max(1024, 2 * N)

    def alloc(c):
        return (torch.empty(c, dtype=torch.int32, device=dev), torch.empty(c, dtype=torch.int32, device=dev),
                torch.empty(c, dtype=torch.float64, device=dev) if nearest else None)

    left, right, dists = alloc(cap)

    def join(l, r, d):
        if nearest:
            return index.nearest_into(pts, l, r, d)
        return index.dwithin_into(pts, l, r, distance=DWITHIN_DISTANCE)

    try:
        n_pairs, st = join(left, right, dists)
    except _abi.CapacityError as e:
        cap = e.required
        left, right, dists = alloc(cap)
        n_pairs, st = join(left, right, dists)
    for _ in range(args.warmup):
        join(left, right, dists)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, launches = [], 0
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            ev[k][0].record(stream)
            n_k, st = join(left, right, dists)
            ev[k][1].record(stream)
            kernel_ms.append(st["kernel_ms"])
            launches += st["kernel_launches"]
            assert n_k == n_pairs
        torch.cuda.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        # e2e: points from pinned host memory, pairs (and distances) back to pinned host memory
        hx = torch.from_numpy(w.px).pin_memory()
        hy = torch.from_numpy(w.py).pin_memory()
        hl = torch.empty(n_pairs, dtype=torch.int32).pin_memory()
        hr = torch.empty(n_pairs, dtype=torch.int32).pin_memory()
        hd = torch.empty(n_pairs, dtype=torch.float64).pin_memory() if nearest else None
        e2e_ms = []
        for k in range(max(3, args.steps) + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            dx.copy_(hx, non_blocking=True)
            dy.copy_(hy, non_blocking=True)
            n_e, _ = join(left, right, dists)
            hl.copy_(left[:n_e], non_blocking=True)
            hr.copy_(right[:n_e], non_blocking=True)
            if nearest:
                hd.copy_(dists[:n_e], non_blocking=True)
            b.record(stream)
            torch.cuda.synchronize()
            if k:
                e2e_ms.append(a.elapsed_time(b))
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms, float(np.median(e2e_ms))], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        total_ms, e2e_med = float(t[0]), float(t[1])
    else:
        e2e_med = float(np.median(e2e_ms))
    # points every rank processed per step: N each (weak), or the one dataset (sharded)
    n_job = w.n_points if sharded else world * N
    value = n_job * args.steps / (total_ms / 1e3)
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    kmed = float(np.median(kernel_ms))
    B = algorithmic_bytes(w, n_pairs) + (8 * n_pairs if nearest else 0)
    achieved = B / (kmed / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / f"traffic_{args.workload}_rtree.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get("traffic_bytes_per_launch")
        except Exception:
            traffic = None
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        rate, n_s, dt = cpu_distance_rate(w, args.workload, threads, args.cpu_seconds)
        cpu = {"value": rate, "unit": "points/s", "cores": threads, "kind": "port",
               "sample": f"first {n_s} of {N} points vs all {len(w.polys)} polygons ({dt:.1f} s), CPU oracle "
                         "(C + OpenMP, grid index, same distance arithmetic); Shapely/GEOS is not installable here"}
    line = {
        "metric": "query points/sec", "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc(args, args.workload), "method": "rtree (distance walk)",
                   "n_points_per_gpu": N, "n_polygons": len(w.polys), "n_pairs": n_pairs,
                   "distance": None if nearest else DWITHIN_DISTANCE,
                   "parallelism": f"points sharded over {world} GPU(s), index replicated",
                   "l2": "inputs (800 MB of points) larger than L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel_ms": kmed,
                     "algorithmic_bytes_per_launch": B},
        "cpu_baseline": cpu,
        "e2e": {"value": world * N / (e2e_med / 1e3), "unit": "points/s",
                "h2d_bytes_per_step": int(16 * N), "d2h_bytes_per_step": int((16 if nearest else 8) * n_pairs)},
        "gpu_launches": launches,
        "join_stats": st,
    }
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def _export_inputs(w, pairs_l, pairs_r):
    n_left, n_right = w.n_points, len(w.polys.geom_off) - 1
    return n_left, n_right, (np.arange(n_left, dtype=np.int64) % 7), (np.arange(n_right, dtype=np.int64) % 7)


def run_reference_export(args, world):
    """The host export (numpy restatement of the reference's _adjust_join_indexers
    and attribute filter) on the same pairs, made by the CPU oracle."""
    import importlib

    sj = importlib.import_module("vibespatial_b200.sjoin")
    w = make_workload("zipf", 0, args.scale)
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    P = O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    hl, hr = O.join(w.px, w.py, None, P, "within", os.cpu_count() or 1)
    n_left, n_right, lc, rc = _export_inputs(w, hl, hr)
    for _ in range(args.warmup):
        out = sj._join_indexers(hl, hr, n_left, n_right, "left", (lc, rc))
    n_rows = len(out[0])
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sj._join_indexers(hl, hr, n_left, n_right, "left", (lc, rc))
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n_rows * len(times) / tot
    line = {
        "impl": "reference", "metric": "join export rows/sec", "value": value, "unit": "rows/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": workload_desc(args, "export"), "n_pairs": int(len(hl)), "n_rows": n_rows},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": 1, "kind": "port",
                         "sample": "the whole export each step: numpy restatement of the reference's host "
                                   "_adjust_join_indexers + attribute filter"},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_export(args, rank, world, local_rank):
    """Join export (vs_join_export) of the zipf within pairs: how='left' + on_attribute codes."""
    import importlib

    import torch

    from vibespatial_b200 import _abi

    sj = importlib.import_module("vibespatial_b200.sjoin")
    dev = local_rank
    torch.cuda.set_device(dev)
    w = make_workload("zipf", rank, args.scale)
    ctx = _abi.Context(dev)
    stream = ctx.torch_stream
    pol = w.polys
    d_poly = {k: torch.from_numpy(np.ascontiguousarray(getattr(pol, k))).to(dev)
              for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    P = _abi.make_polygons(d_poly["x"], d_poly["y"], d_poly["ring_off"], d_poly["part_off"], d_poly["geom_off"])
    index = _abi.DeviceIndex(ctx, P, learned=True)
    dx, dy = torch.from_numpy(w.px).to(dev), torch.from_numpy(w.py).to(dev)
    pts = _abi.make_points(dx, dy)
    left, right, _ = index.join(pts, _abi.PRED_WITHIN, _abi.METHOD_LEARNED, sort=True)
    n_left, n_right, lc_h, rc_h = _export_inputs(w, left, right)
    lc, rc = torch.from_numpy(lc_h).to(dev), torch.from_numpy(rc_h).to(dev)

    def step():
        return _abi.join_export(ctx, left, right, n_left, n_right, "left", lc, rc)

    out = step()
    n_rows = int(out[0].numel())
    # the device rows equal the host export of the same pairs
    hl, hr = left.cpu().numpy(), right.cpu().numpy()
    el, er, es = sj._join_indexers(hl, hr, n_left, n_right, "left", (lc_h, rc_h))
    assert np.array_equal(out[0].cpu().numpy(), el) and np.array_equal(out[1].cpu().numpy(), er)
    assert np.array_equal(out[2].cpu().numpy(), es)
    del out
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = _abi.kernel_launches()
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        launches = _abi.kernel_launches() - launches0
        # e2e: pairs and codes from pinned host memory, the three indexers back to pinned host memory
        h_l, h_r = torch.from_numpy(hl).pin_memory(), torch.from_numpy(hr).pin_memory()
        h_lc, h_rc = torch.from_numpy(lc_h).pin_memory(), torch.from_numpy(rc_h).pin_memory()
        o = [torch.empty(n_rows, dtype=torch.int64).pin_memory() for _ in range(3)]
        e2e_ms = []
        for k in range(max(3, args.steps) + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            dl, dr = h_l.to(dev, non_blocking=True), h_r.to(dev, non_blocking=True)
            dlc, drc = h_lc.to(dev, non_blocking=True), h_rc.to(dev, non_blocking=True)
            res = _abi.join_export(ctx, dl, dr, n_left, n_right, "left", dlc, drc)
            for t, d in zip(o, res):
                t.copy_(d, non_blocking=True)
            b.record(stream)
            torch.cuda.synchronize()
            if k:
                e2e_ms.append(a.elapsed_time(b))
    total_ms = float(sum(step_ms))
    value = n_rows * args.steps / (total_ms / 1e3)
    e2e_med = float(np.median(e2e_ms))
    peak, peak_kind = _peaks()
    n_pairs = int(left.numel())
    # algorithmic bytes: pairs (8) + their two codes (16) read, kept pairs re-read, output rows (24) written,
    # per-left-row counts (4 + 4 read) -- the minimum of a filter-then-expand export
    B = 8 * n_pairs + 16 * n_pairs + 24 * n_rows + 8 * n_left
    kmed = float(np.median(step_ms))
    achieved = B / (kmed / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < min(args.cpu_seconds, 10.0) or reps == 0:
            sj._join_indexers(hl, hr, n_left, n_right, "left", (lc_h, rc_h))
            reps += 1
        dt = time.perf_counter() - t0
        cpu = {"value": n_rows * reps / dt, "unit": "rows/s", "cores": 1, "kind": "port",
               "sample": f"the whole export, {reps} time(s) ({dt:.1f} s): numpy restatement of the reference's "
                         "host _adjust_join_indexers + attribute filter"}
    line = {
        "metric": "join export rows/sec", "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": workload_desc(args, "export"), "n_pairs": n_pairs, "n_left": n_left, "n_right": n_right,
                   "n_rows": n_rows, "how": "left", "l2": "inputs (~0.6 GB) larger than L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel_ms": kmed, "algorithmic_bytes_per_launch": B},
        "cpu_baseline": cpu,
        "e2e": {"value": n_rows / (e2e_med / 1e3), "unit": "rows/s",
                "h2d_bytes_per_step": int(8 * n_pairs + 8 * (n_left + n_right)),
                "d2h_bytes_per_step": int(24 * n_rows)},
        "gpu_launches": launches,
    }
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def run_reference_nearest_polygons(args, world):
    """The CPU oracle (brute force over the points with the envelope bound, all
    host threads) on the first polygons of the same workload."""
    w = make_workload("zipf", 0, args.scale)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    pol = w.polys
    k = 32
    SP = O.Polygons(pol.x, pol.y, pol.ring_off, pol.part_off, pol.geom_off[:k + 1])
    for _ in range(args.warmup):
        O.nearest_polygons_join(w.px, w.py, None, SP, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.nearest_polygons_join(w.px, w.py, None, SP, threads=threads)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = k * len(times) / tot
    line = {
        "impl": "reference", "metric": "query polygons/sec", "value": value, "unit": "polygons/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc(args, "nearest_polygons"), "sample_polygons": k, "n_points": w.n_points},
        "cpu_baseline": {"value": value, "unit": "polygons/s", "cores": threads, "kind": "port",
                         "sample": f"the first {k} polygons against all {w.n_points} points each step, CPU oracle "
                                   "(C + OpenMP); Shapely/GEOS is not installable here"},
        "e2e": {"value": value, "unit": "polygons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_nearest_polygons(args, rank, world, local_rank):
    """Nearest points of every polygon through vs_join_nearest_polygons (index over the points)."""
    import torch

    from vibespatial_b200 import _abi

    dev = local_rank
    torch.cuda.set_device(dev)
    w = make_workload("zipf", rank, args.scale)
    ctx = _abi.Context(dev)
    stream = ctx.torch_stream
    pol = w.polys
    d_poly = {k: torch.from_numpy(np.ascontiguousarray(getattr(pol, k))).to(dev)
              for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    P = _abi.make_polygons(d_poly["x"], d_poly["y"], d_poly["ring_off"], d_poly["part_off"], d_poly["geom_off"])
    dx, dy = torch.from_numpy(w.px).to(dev), torch.from_numpy(w.py).to(dev)
    t0 = time.perf_counter()
    pidx = _abi.point_index(ctx, dx, dy)
    build_wall = time.perf_counter() - t0
    M = len(pol.geom_off) - 1
    left, _, _, st = _abi.nearest_polygons(ctx, pidx, P)
    n_pairs = int(left.numel())
    cap = max(n_pairs, 1)
    for _ in range(args.warmup):
        _abi.nearest_polygons(ctx, pidx, P, capacity=cap)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, launches = [], 0
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            ev[k][0].record(stream)
            _, _, _, st = _abi.nearest_polygons(ctx, pidx, P, capacity=cap)
            ev[k][1].record(stream)
            kernel_ms.append(st["kernel_ms"])
            launches += st["kernel_launches"]
        torch.cuda.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    value = M * args.steps / (total_ms / 1e3)
    peak, peak_kind = _peaks()
    kmed = float(np.median(kernel_ms))
    B = algorithmic_bytes(w, n_pairs) + 8 * n_pairs
    achieved = B / (kmed / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        O.build()
        threads = os.cpu_count() or 1
        k = 64
        sub = {"x": pol.x, "y": pol.y, "ring_off": pol.ring_off, "part_off": pol.part_off,
               "geom_off": pol.geom_off[:k + 1]}
        SP = O.Polygons(sub["x"], sub["y"], sub["ring_off"], sub["part_off"], sub["geom_off"])
        t0 = time.perf_counter()
        O.nearest_polygons_join(w.px, w.py, None, SP, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": k / dt, "unit": "polygons/s", "cores": threads, "kind": "port",
               "sample": f"the first {k} of {M} polygons against all {w.n_points} points ({dt:.1f} s), CPU oracle "
                         "(C + OpenMP, brute force over the points with the envelope bound)"}
    line = {
        "metric": "query polygons/sec", "value": value, "unit": "polygons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc(args, "nearest_polygons"), "n_polygons": M, "n_points": w.n_points,
                   "n_pairs": n_pairs, "point_index_build_wall_s": build_wall,
                   "l2": "inputs (800 MB of points, index 1.6 GB) larger than L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel_ms": kmed, "algorithmic_bytes_per_launch": B},
        "cpu_baseline": cpu,
        "e2e": None,
        "gpu_launches": launches,
        "join_stats": st,
    }
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload == "batched":
        run_reference_batched(args, world)
        return
    if args.workload == "wkb":
        run_reference_wkb(args, world)
        return
    if args.workload in ("dwithin", "nearest"):
        run_reference_distance(args, world)
        return
    if args.workload == "export":
        run_reference_export(args, world)
        return
    if args.workload == "nearest_polygons":
        run_reference_nearest_polygons(args, world)
        return
    w = make_workload(args.workload, 0, args.scale)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.build()
    P = O.Polygons(w.polys.x, w.polys.y, w.polys.ring_off, w.polys.part_off, w.polys.geom_off)
    # a strided sample (every stride-th point), so that it follows the whole
    # workload's distribution (every Zipf site, every cluster) rather than a prefix
    stride = max(1, -(-w.n_points // max(1, args.ref_sample)))
    sx, sy = np.ascontiguousarray(w.px[::stride]), np.ascontiguousarray(w.py[::stride])
    n = len(sx)
    for _ in range(args.warmup):
        O.join(sx, sy, None, P, args.predicate, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.join(sx, sy, None, P, args.predicate, threads)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * len(times) / tot
    line = {
        "impl": "reference", "metric": "query points/sec", "value": value, "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": join_config(args, w),
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads, "kind": "port",
                         "sample": f"{every(stride, 'point')} ({n} of {w.n_points}) vs all {len(w.polys)} polygons, "
                                   "exact CPU oracle (C + OpenMP): Shapely/GEOS is not installable here",
                         "shapely_importable": shapely_importable()},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch

    from vibespatial_b200 import _abi

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = world > 1
    if dist:
        import torch.distributed as tdist

    # default: every rank joins a dataset of its own (weak scaling); with
    # --shard hilbert all ranks hold one dataset and each joins its
    # Hilbert-range shard of the points (strong scaling), pairs assembled on rank 0
    sharded = args.shard == "hilbert"
    w = make_workload(args.workload, 0 if sharded else rank, args.scale)
    rows = None
    px, py = w.px, w.py
    if sharded:
        from vibespatial_b200.sharding import hilbert_shard_rows

        rows = hilbert_shard_rows(w.px, w.py, rank, world)
        px, py = np.ascontiguousarray(w.px[rows]), np.ascontiguousarray(w.py[rows])
    N = len(px)
    ctx = _abi.Context(dev)
    stream = ctx.torch_stream
    pol = w.polys
    d_poly = {k: torch.from_numpy(np.ascontiguousarray(getattr(pol, k))).to(dev)
              for k in ("x", "y", "ring_off", "part_off", "geom_off")}
    P = _abi.make_polygons(d_poly["x"], d_poly["y"], d_poly["ring_off"], d_poly["part_off"], d_poly["geom_off"])
    method = _abi.METHOD_RTREE if args.method == "rtree" else _abi.METHOD_LEARNED
    batched = args.method == "learned-batched"
    pred = {"within": _abi.PRED_WITHIN, "intersects": _abi.PRED_INTERSECTS}[args.predicate]
    t0 = time.perf_counter()
    index = _abi.DeviceIndex(ctx, P, learned=(method == _abi.METHOD_LEARNED), ring_bin_min_vertices=args.ring_bin_min,
                             cell_level=args.cell_level)
    build_wall = time.perf_counter() - t0
    info = index.info()
    del d_poly
    dx = torch.from_numpy(px).to(dev)
    dy = torch.from_numpy(py).to(dev)
    pts = _abi.make_points(dx, dy)
    # size the pair buffers once (exact count from a first join)
    cap = max(1024, N)
    left = torch.empty(cap, dtype=torch.int32, device=dev)
    right = torch.empty(cap, dtype=torch.int32, device=dev)
    try:
        n_pairs, _ = index.join_into(pts, pred, method, left, right)
    except _abi.CapacityError as e:
        cap = e.required
        left = torch.empty(cap, dtype=torch.int32, device=dev)
        right = torch.empty(cap, dtype=torch.int32, device=dev)
        n_pairs, _ = index.join_into(pts, pred, method, left, right)
    plan = None
    plan_opts, plan_opts_src = None, None
    if batched:
        # learned + batched: the join as a one-job batch plan (the persistent
        # learned pipeline replayed from a CUDA graph), its launch shape from the
        # autotuner (cached, else searched now, before any timing)
        from vibespatial_b200 import autotune

        plan_opts, plan_opts_src = autotune.tuned_options(
            ctx, [index], pts, [0, N], pred, len(w.polys), left=left, right=right, use_cache=not args.autotune,
            method=_abi.METHOD_LEARNED, with_source=True)
        plan = _abi.BatchPlan(ctx, [index], pts, [0, N], options=dict(plan_opts, method=_abi.METHOD_LEARNED))

    def join(lft, rgt):
        if plan is not None:
            return plan.run_into(pred, lft, rgt, use_graph=True)
        return index.join_into(pts, pred, method, lft, rgt)

    assembled = {}

    def assemble(lft, rgt, n_local):
        """Sharded mode, N > 1: every rank's pairs (shard-local point rows)
        sent to rank 0 over NCCL, sized by an all-gather of the counts."""
        with torch.cuda.stream(stream):
            cnt = torch.tensor([n_local], dtype=torch.int64, device=dev)
            allc = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
            tdist.all_gather(allc, cnt)
            counts = [int(c.item()) for c in allc]
            if rank == 0:
                if "l" not in assembled:
                    assembled["l"] = torch.empty(max(1, sum(counts)), dtype=torch.int32, device=dev)
                    assembled["r"] = torch.empty(max(1, sum(counts)), dtype=torch.int32, device=dev)
                off = counts[0]
                for r in range(1, world):
                    if counts[r]:
                        tdist.recv(assembled["l"][off:off + counts[r]], src=r)
                        tdist.recv(assembled["r"][off:off + counts[r]], src=r)
                    off += counts[r]
            elif n_local:
                tdist.send(lft[:n_local], dst=0)
                tdist.send(rgt[:n_local], dst=0)
        return counts

    assert join(left, right)[0] == n_pairs
    # plain R-tree on the same GPU, for the learned-vs-plain ratio
    plain = None
    if method == _abi.METHOD_LEARNED:
        n_plain, _ = index.join_into(pts, pred, _abi.METHOD_RTREE, left, right)
        assert n_plain == n_pairs, (n_plain, n_pairs)

    for _ in range(args.warmup):
        n_w, _ = join(left, right)
        if sharded and dist:
            assemble(left, right, n_w)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, phases = [], []
    launches = 0
    plain_phases = None
    with ClockSampler(dev) as clk:
        if args.profile:
            torch.cuda.profiler.start()  # ncu --profile-from-start off captures the timed steps only
        for k in range(args.steps):
            ev[k][0].record(stream)
            n_k, st = join(left, right)
            if sharded and dist:
                assemble(left, right, n_k)
            ev[k][1].record(stream)
            kernel_ms.append(st["kernel_ms"])
            phases.append(st["phase_ms"])
            launches += st["kernel_launches"]
            assert n_k == n_pairs
        torch.cuda.synchronize()
        if args.profile:
            torch.cuda.profiler.stop()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        # plain method timing (same GPU, same buffers) after the timed region
        if method == _abi.METHOD_LEARNED:
            pm, pph = [], []
            for _ in range(max(3, args.steps // 2)):
                _, stp = index.join_into(pts, pred, _abi.METHOD_RTREE, left, right)
                pm.append(stp["kernel_ms"])
                pph.append(stp["phase_ms"])
            plain = float(np.median(pm))
            plain_phases = [float(v) for v in np.median(np.array(pph), axis=0)]
            # the plain traversal with leaf blocks by bulk copies (TMA)
            pb = []
            for _ in range(max(3, args.steps // 2)):
                _, stb = index.join_into(pts, pred, _abi.METHOD_RTREE, left, right, flags=_abi.JOIN_BULK_LEAVES)
                pb.append(stb["kernel_ms"])
            plain_bulk = float(np.median(pb))
        ablations = None
        if batched:
            # per-phase device times of the same learned pipeline, launched
            # directly (a graph replay records no phase marks)
            dph = []
            for _ in range(max(3, args.steps // 2)):
                dph.append(index.join_into(pts, pred, _abi.METHOD_LEARNED, left, right)[1]["phase_ms"])
            phases = dph
            ablations = learned_ablations(_abi, ctx, [index], pts, [0, N], pred, left, right, n_pairs,
                                          dict(plan_opts, method=_abi.METHOD_LEARNED), max(3, args.steps // 2))
            if plain is not None:
                ablations["plain_rtree_ms"] = plain
        # e2e through the C-ABI with HOST buffers (vs_join_host): pinned host
        # points in, pinned host pairs out, the chunked copies overlapping the join
        hx = torch.from_numpy(px).pin_memory()
        hy = torch.from_numpy(py).pin_memory()
        hl = torch.empty(cap, dtype=torch.int32).pin_memory()
        hr = torch.empty(cap, dtype=torch.int32).pin_memory()
        e2e_ms = []
        for k in range(max(3, args.steps) + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            n_e, _ = index.join_host(hx, hy, pred, method, hl, hr)
            b.record(stream)
            torch.cuda.synchronize()
            assert n_e == n_pairs, (n_e, n_pairs)
            if k:  # the first call warms the host pipeline
                e2e_ms.append(a.elapsed_time(b))
    # the pairs of the benchmarked call and of the e2e call, kept for the check
    # against the CPU oracle below (outside every timed region)
    n_chk, _ = join(left, right)
    gl_chk, gr_chk = left[:n_chk].clone(), right[:n_chk].clone()
    if n_chk:
        _abi.sort_pairs(ctx, gl_chk, gr_chk)
    gl_chk, gr_chk = gl_chk.cpu().numpy(), gr_chk.cpu().numpy()
    hl_chk, hr_chk = hl[:n_e].numpy().copy(), hr[:n_e].numpy().copy()
    if rows is not None:  # shard-local point rows -> the dataset's rows
        gl_chk, hl_chk = rows[gl_chk], rows[hl_chk]
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms, float(np.median(e2e_ms))], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        total_ms, e2e_med = float(t[0]), float(t[1])
    else:
        e2e_med = float(np.median(e2e_ms))
    # points every rank processed per step: N each (weak), or the one dataset (sharded)
    n_job = w.n_points if sharded else world * N
    value = n_job * args.steps / (total_ms / 1e3)
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    kmed = float(np.median(kernel_ms))
    B = algorithmic_bytes(w, n_pairs, N)
    achieved = B / (kmed / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / f"traffic_{args.workload}_{args.method}.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get("traffic_bytes_per_launch")
        except Exception:
            traffic = None
    cpu = None
    parity = None
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        rate, n_s, dt, cpu_pairs = cpu_sample_rate(w, args.predicate, threads, args.cpu_seconds)
        cpu = {"value": rate, "unit": "points/s", "cores": threads, "kind": "port",
               "sample": f"first {n_s} of {N} points vs all {len(w.polys)} polygons ({dt:.1f} s), exact CPU "
                         "oracle (C + OpenMP); Shapely/GEOS is not installable here",
               "shapely_importable": shapely_importable()}
        if cpu_pairs is not None:
            parity = {"checker": "exact CPU oracle, all points", "oracle_pairs": int(len(cpu_pairs[0])),
                      "mismatches": pair_mismatches(gl_chk, gr_chk, *cpu_pairs),
                      "e2e_mismatches": pair_mismatches(hl_chk, hr_chk, *cpu_pairs)}
    e32, e64 = st.get("fp32_edges", 0), st.get("fp64_edges", 0)
    line = {
        "metric": "query points/sec", "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": join_config(args, w),
        "method": args.method, "n_pairs": n_pairs,
        "parallelism": (f"one dataset, Hilbert-range shards of the points over {world} GPU(s), index replicated, "
                        "pairs assembled on rank 0 (NCCL send/recv) every step" if sharded else
                        f"points sharded over {world} GPU(s), index replicated"),
        "index": {"build_ms": info["build_ms"], "build_wall_s": build_wall, "device_bytes": info["device_bytes"]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel_ms": kmed,
                     "algorithmic_bytes_per_launch": B},
        "cpu_baseline": cpu,
        "parity": parity,
        "split_precision": {"fp32_edges": e32, "fp64_edges": e64,
                            "fp32_pass_rate": (e32 / (e32 + e64)) if e32 + e64 else None,
                            "exact_fallbacks": st.get("exact_fallbacks", 0)},
        "e2e": {"value": n_job / (e2e_med / 1e3), "unit": "points/s",
                "h2d_bytes_per_step": int(16 * N), "d2h_bytes_per_step": int(8 * n_pairs)},
        "gpu_launches": launches,
        "phases_ms": dict(zip(PHASES, (float(v) for v in np.median(np.array(phases), axis=0)))),
        "join_stats": st,
        "index_info": info,
    }
    if ablations is not None:
        line["ablations"] = ablations
    if plan_opts is not None:
        line["launch_shape"] = plan_opts
        line["launch_shape_source"] = plan_opts_src
    if plain is not None:
        line["plain_rtree_ms"] = plain
        line["plain_rtree_bulk_leaves_ms"] = plain_bulk
        line["plain_phases_ms"] = dict(zip(PHASES, plain_phases))
        line["learned_vs_plain"] = plain / kmed
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def run_batched(args, rank, world, local_rank):
    """Batched joins: all jobs in one persistent launch, replayed from a CUDA graph."""
    import torch

    from vibespatial_b200 import _abi, autotune

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
    jobs = make_batched(rank, args.scale)
    learned = args.method != "rtree"
    bmethod = _abi.METHOD_LEARNED if learned else _abi.METHOD_RTREE
    ctx = _abi.Context(dev)
    stream = ctx.torch_stream
    pred = {"within": _abi.PRED_WITHIN, "intersects": _abi.PRED_INTERSECTS}[args.predicate]
    t0 = time.perf_counter()
    indexes, build_ms, n_polys = [], 0.0, 0
    for w in jobs:
        d = {k: torch.from_numpy(np.ascontiguousarray(getattr(w.polys, k))).to(dev)
             for k in ("x", "y", "ring_off", "part_off", "geom_off")}
        ix = _abi.DeviceIndex(ctx, _abi.make_polygons(d["x"], d["y"], d["ring_off"], d["part_off"], d["geom_off"]),
                              learned=learned, ring_bin_min_vertices=args.ring_bin_min)
        indexes.append(ix)
        build_ms += ix.info()["build_ms"]
        n_polys += len(w.polys)
    build_wall = time.perf_counter() - t0
    px = np.concatenate([w.px for w in jobs])
    py = np.concatenate([w.py for w in jobs])
    job_start = np.concatenate([[0], np.cumsum([w.n_points for w in jobs])]).astype(np.int64)
    N = len(px)
    dx = torch.from_numpy(px).to(dev)
    dy = torch.from_numpy(py).to(dev)
    pts = _abi.make_points(dx, dy)
    # exact pair count from a first direct run, then buffers of that size
    probe = _abi.BatchPlan(ctx, indexes, pts, job_start, options={"method": bmethod})
    probe_l, _, _ = probe.run(pred, use_graph=False)
    n_pairs = int(probe_l.numel())
    del probe_l
    probe.close()
    cap = max(1024, n_pairs)
    left = torch.empty(cap, dtype=torch.int32, device=dev)
    right = torch.empty(cap, dtype=torch.int32, device=dev)
    name, sms = autotune.device_identity(dev)
    key = autotune.cache_key(name, sms, autotune.shape_class(len(jobs), N, n_polys), pred)
    # launch shape of the timed plan: the autotuner's (cached, else searched
    # now, before the timed region); --autotune forces a fresh search
    t1 = time.perf_counter()
    opts, opts_src = autotune.tuned_options(ctx, indexes, pts, job_start, pred, n_polys, left=left, right=right,
                                            use_cache=not args.autotune, method=bmethod, with_source=True)
    tune_s = time.perf_counter() - t1
    plan = _abi.BatchPlan(ctx, indexes, pts, job_start, options=dict(opts, method=bmethod))
    for _ in range(args.warmup):
        n_w, _ = plan.run_into(pred, left, right, use_graph=True)
        assert n_w == n_pairs, (n_w, n_pairs)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, launches = [], 0
    with ClockSampler(dev) as clk:
        if args.profile:
            torch.cuda.profiler.start()
        for k in range(args.steps):
            ev[k][0].record(stream)
            n_k, st = plan.run_into(pred, left, right, use_graph=True)
            ev[k][1].record(stream)
            kernel_ms.append(st["kernel_ms"])
            launches += st["kernel_launches"]
            assert n_k == n_pairs
        torch.cuda.synchronize()
        if args.profile:
            torch.cuda.profiler.stop()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        # the R-tree batch on the same jobs, for the learned-vs-plain ratio
        rtree_batch_ms = None
        ablations = None
        if learned:
            ropts = autotune.tuned_options(ctx, indexes, pts, job_start, pred, n_polys, left=left, right=right,
                                           use_cache=not args.autotune, method=_abi.METHOD_RTREE)
            rplan = _abi.BatchPlan(ctx, indexes, pts, job_start, options=dict(ropts, method=_abi.METHOD_RTREE))
            rms = []
            for k in range(3 + max(3, args.steps // 2)):
                n_r, st_r = rplan.run_into(pred, left, right, use_graph=True)
                assert n_r == n_pairs, (n_r, n_pairs)
                if k >= 3:
                    rms.append(st_r["kernel_ms"])
            rplan.close()
            rtree_batch_ms = float(np.median(rms))
            ablations = learned_ablations(_abi, ctx, indexes, pts, job_start, pred, left, right, n_pairs,
                                          dict(opts, method=bmethod), max(3, args.steps // 2))
            ablations["plain_rtree_batched_ms"] = rtree_batch_ms
        # the same jobs one vs_join call at a time (how a caller without the
        # batch API runs them), after the timed region
        loop_ms = []
        views = [(_abi.make_points(dx[a:b], dy[a:b]), a) for a, b in zip(job_start[:-1], job_start[1:])]
        for _ in range(3):
            a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a_ev.record(stream)
            off = 0
            for ix, (pv, _a) in zip(indexes, views):
                n_j, _ = ix.join_into(pv, pred, bmethod, left[off:], right[off:])
                off += n_j
            b_ev.record(stream)
            torch.cuda.synchronize()
            assert off == n_pairs, (off, n_pairs)
            loop_ms.append(a_ev.elapsed_time(b_ev))
        # e2e through the C-ABI with host buffers: H2D points, batched join, D2H pairs
        hx = torch.from_numpy(px).pin_memory()
        hy = torch.from_numpy(py).pin_memory()
        hl = torch.empty(cap, dtype=torch.int32).pin_memory()
        hr = torch.empty(cap, dtype=torch.int32).pin_memory()
        e2e_ms = []
        for _ in range(max(3, args.steps)):
            a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                a_ev.record(stream)
                dx.copy_(hx, non_blocking=True)
                dy.copy_(hy, non_blocking=True)
                n_e, _ = plan.run_into(pred, left, right, use_graph=True)
                assert n_e == n_pairs, (n_e, n_pairs)
                hl[:n_e].copy_(left[:n_e], non_blocking=True)
                hr[:n_e].copy_(right[:n_e], non_blocking=True)
                b_ev.record(stream)
            torch.cuda.synchronize()
            e2e_ms.append(a_ev.elapsed_time(b_ev))
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms, float(np.median(e2e_ms))], device=dev, dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        total_ms, e2e_med = float(t[0]), float(t[1])
    else:
        e2e_med = float(np.median(e2e_ms))
    value = world * N * args.steps / (total_ms / 1e3)
    plan.close()
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    kmed = float(np.median(kernel_ms))
    B = sum(algorithmic_bytes(w, 0) for w in jobs) + 8 * n_pairs
    achieved = B / (kmed / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / f"traffic_batched_{'learned' if learned else 'rtree'}.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get("traffic_bytes_per_launch")
        except Exception:
            traffic = None
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        rate, n_s, dt, k = cpu_sample_batched(jobs, args.predicate, threads, args.cpu_seconds)
        cpu = {"value": rate, "unit": "points/s", "cores": threads, "kind": "port",
               "sample": f"first {k} of {len(jobs)} jobs ({n_s} points, {dt:.1f} s), exact CPU oracle "
                         "(C + OpenMP); Shapely/GEOS is not installable here"}
    loop_med = float(np.median(loop_ms))
    line = {
        "metric": "query points/sec", "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": batched_config(args, jobs),
        "method": ("learned" if learned else "rtree") + ", batched", "n_pairs": n_pairs,
        "parallelism": f"jobs replicated per GPU ({world} GPU(s)), independent",
        "launch_shape": opts, "launch_shape_source": opts_src, "autotune_s": tune_s,
        "index": {"build_ms": build_ms, "build_wall_s": build_wall},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel_ms": kmed,
                     "algorithmic_bytes_per_launch": B},
        "cpu_baseline": cpu,
        "e2e": {"value": world * N / (e2e_med / 1e3), "unit": "points/s",
                "h2d_bytes_per_step": int(16 * N), "d2h_bytes_per_step": int(8 * n_pairs)},
        "gpu_launches": launches,
        "join_stats": st,
        "per_job_loop_ms": loop_med,
        "batched_vs_loop": loop_med / kmed,
    }
    if ablations is not None:
        line["ablations"] = ablations
    if rtree_batch_ms is not None:
        line["plain_rtree_batched_ms"] = rtree_batch_ms
        line["learned_vs_plain"] = rtree_batch_ms / kmed
    line["clocks"] = clk.summary()
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOAD_DESC), default="zipf")
    ap.add_argument("--predicate", choices=["within", "intersects"], default="within")
    ap.add_argument("--method", choices=["learned-batched", "learned", "rtree"], default="learned-batched",
                    help="learned-batched: the learned pipeline as a batch plan replayed from a CUDA graph; "
                         "learned: vs_join with the learned index; rtree: the plain R-tree traversal")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-sample", type=int, default=4_000_000)
    ap.add_argument("--shard", choices=["none", "hilbert"], default="none",
                    help="none: each rank joins its own dataset (weak scaling); hilbert: one dataset, each rank "
                         "joins a Hilbert-range shard of its points and rank 0 assembles the pairs (strong scaling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ring-bin-min", type=int, default=0,
                    help="rings with at least this many vertices get y-bins (0: library default, <0: none)")
    ap.add_argument("--cell-level", type=int, default=0,
                    help="learned index grid level of the join workloads (0: automatic); a scaled-down profiling "
                         "run can keep the full-size workload's level")
    ap.add_argument("--autotune", action="store_true",
                    help="batched workload: search the launch shape now instead of using the cache/defaults")
    ap.add_argument("--profile", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                 device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "batched":
            run_batched(args, rank, world, local_rank)
        elif args.workload == "wkb":
            run_wkb(args, rank, world, local_rank)
        elif args.workload in ("dwithin", "nearest"):
            run_distance(args, rank, world, local_rank)
        elif args.workload == "export":
            run_export(args, rank, world, local_rank)
        elif args.workload == "nearest_polygons":
            run_nearest_polygons(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist

            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
