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


def test_every_profile_the_bench_reads_carries_its_traffic():
    """Each ncu summary bench.py reads a roofline traffic figure from exists
    under profiles/ and carries the machine-read lines, so no workload
    record's `traffic` silently turns null after a summary is renamed."""
    import re
    sys.path.insert(0, str(ROOT))
    import bench
    names = set(re.findall(r'traffic_per_launch\("([^"]+)"', (ROOT / "bench.py").read_text()))
    names.add("selective_scan_sum_60M_scan_kernel.md")   # the headline's default
    assert len(names) >= 4
    for name in sorted(names):
        assert (ROOT / "profiles" / name).exists(), name
        t = bench.traffic_per_launch(name)
        assert t is not None and t > 0, name
        text = (ROOT / "profiles" / name).read_text()
        if "captured_rows:" in text:
            assert bench.traffic_per_launch(name, 2 * int(re.search(r"captured_rows:\s*(\d+)", text).group(1))) == \
                   2 * t
