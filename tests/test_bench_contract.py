"""bench.py's reference arm runs on CPU: its JSON line carries the keys the
benchmark contract names, for the default workload and a grouped one, and the
workloads without a CPU counterpart print the unavailable line."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def run(*args):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def check_line(d):
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "rows/s"
    assert d["higher_is_better"] is True and d["warmup"] >= 3
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_default_workload():
    d = run("--steps", "1", "--warmup", "3", "--reference-rows", "300000")
    check_line(d)
    assert d["config"]["workload"].startswith("selective_scan_sum")


def test_reference_arm_grouped_workload():
    d = run("--workload", "filtered_group_agg", "--steps", "1", "--warmup", "3", "--rows", "400000")
    check_line(d)
    assert d["config"]["workload"].startswith("filtered_group_agg (400000 rows")


def test_reference_arm_join_and_highcard_workloads():
    for w in ("join_group_agg", "highcard_group"):
        d = run("--workload", w, "--steps", "1", "--warmup", "3", "--rows", "300000")
        check_line(d)
        assert d["config"]["workload"].startswith(w) and d["cpu_baseline"]["cores"] >= 1
        assert "restatement of the reference's" in d["cpu_baseline"]["sample"]


def test_reference_arm_unavailable_for_serving():
    for w in ("batch", "serve"):
        d = run("--workload", w, "--steps", "1", "--warmup", "3")
        assert d["impl"] == "reference" and "unavailable" in d
