"""bench.py's reference arm (the CPU oracle timed on the host cores) prints
exactly one JSON line with the contract's keys, on the GPU arm's metric,
unit and configuration; run here at a small scale so it takes seconds."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup",
                          "3", "--scale", "0.01", "--cpu-seconds", "1"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert (d["metric"], d["unit"], d["higher_is_better"]) == ("query points/sec", "points/s", True)
    assert d["steps"] == 1 and d["warmup"] == 3 and d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    # the configuration is the GPU arm's: same keys, and a scaled run says so
    assert set(d["config"]) == {"workload", "predicate", "n_points_per_gpu", "n_polygons", "l2"}
    assert d["config"]["workload"].endswith("(scaled by 0.01)")
    assert d["config"]["n_points_per_gpu"] == 500_000 and d["config"]["n_polygons"] == 10_000


def test_sample_wording():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.every(1, "point") == "every point"
    assert bench.every(2, "job") == "every 2nd job"
    assert bench.every(13, "point") == "every 13th point"
    assert bench.every(21, "point") == "every 21st point"
    assert bench.every(112, "point") == "every 112th point"
