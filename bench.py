"""Benchmark of the hot path.

Headline (default) workload, one step: WHERE ship_day in a 365-day window AND
discount_pct BETWEEN 5 AND 7 AND quantity < 24 → sum(price_cents *
discount_pct) as exact int128, plus count, over 60M seeded synthetic rows
(TPC-H Q6 shape; the data set itself is not available, so seeded columns with
its distributions stand in).

* ``value``  — rows/s with the table resident in HBM (K calls of tgp_execute,
  CUDA events on the library's stream, max over ranks).
* ``e2e``    — rows/s through the C ABI from pinned HOST buffers: every step
  copies the four columns host→device (tgp_table_reload) and reads the result
  back (tgp_execute).
* ``roofline`` — the scan kernel's algorithmic bytes (20 B/row) per launch ÷
  its CUDA-event duration, against the measured HBM copy bandwidth.
* ``cpu_baseline`` — the C++ restatement of the reference's CPU path on this
  host's cores, on a bounded sample of the same workload.
* ``workloads`` — at N=1, one record each for the other workloads at their
  full sizes (filtered grouped aggregate 6M rows, join + grouped aggregate
  60M x 1.5M rows, GROUP BY key over 100M rows, a batch of 256 uneven
  queries, serving against the plain per-query path), with the same keys;
  each record's CPU leg checks the GPU result against the exact checker
  before its numbers are reported.

``--impl reference`` times that CPU restatement alone (rank 0) and prints its
own line (with the same ``config``). Under torchrun, each rank scans its own
60M-row shard (weak scaling); per-step partial sums are merged with an NCCL
all-gather.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ROWS = 60_000_000
BYTES_PER_ROW = 20  # ship_day 4 + discount_pct 4 + quantity 4 + price_cents 8
METRIC = "rows/s & HBM GB/s vs 8 TB/s; batched QPS at p99 vs plain per-query launch"
SCAN_COLUMNS = ("ship_day", "discount_pct", "quantity", "price_cents")
L2_NOTE = "inputs 1.2 GB per rank > 126 MB L2 (no flush needed)"
DATA = "synthetic (seeded; TPC-H lineitem shapes)"
# Full sizes of the other workloads (rows of the scanned / probed table).
FULL_ROWS = {"filtered_group_agg": 6_000_000, "join_group_agg": 60_000_000, "highcard_group": 100_000_000}
DIM_ROWS = 1_500_000


def headline_config(world: int, rows: int) -> dict:
    """The headline line's config, identical in both arms."""
    return {"workload": "selective_scan_sum (60M-row scan, 1.81% selectivity, int128 sum)",
            "rows_per_step": rows, "bytes_per_row": BYTES_PER_ROW, "l2": L2_NOTE,
            "parallelism": f"row shards x{world}"}


def workload_desc(name: str, n: int) -> str:
    if name == "filtered_group_agg":
        return f"filtered_group_agg ({n} rows, WHERE ship_day <= max-90, GROUP BY flag_a, flag_b, 6 aggregates)"
    if name == "join_group_agg":
        return (f"join_group_agg (build {DIM_ROWS} rows filtered on order_day < median, probe {n} rows, "
                f"Zipf(0.8) fk, GROUP BY segment, sum(price*(100-disc)) + count)")
    return f"highcard_group ({n} rows, GROUP BY key Zipf(1.1) over 10M values, count + sum(value))"


def workload_config(name: str, n: int) -> dict:
    """A workload line's config, identical in both arms."""
    per_row = {"filtered_group_agg": 26, "join_group_agg": 16, "highcard_group": 12}[name]
    extra = 9 * DIM_ROWS if name == "join_group_agg" else 0
    b = per_row * n + extra
    return {"workload": workload_desc(name, n), "rows_per_step": n + (DIM_ROWS if name == "join_group_agg" else 0),
            "bytes_per_step": b, "l2": "inputs larger than the 126 MB L2" if b > 126e6 else "inputs smaller than L2"}


def peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def traffic_per_launch(profile: str = "selective_scan_sum_60M_scan_kernel.md", rows: int | None = None) -> float | None:
    """DRAM bytes (read + write) per launch from a committed ncu summary, if
    present; with ``rows``, scaled from the captured row count (the summary
    says where its traffic grows in proportion to the rows)."""
    p = ROOT / "profiles" / profile
    if not p.exists():
        return None
    vals = {}
    for line in p.read_text().splitlines():
        for k in ("traffic_bytes_per_launch:", "captured_rows:"):
            if line.startswith(k):
                vals[k] = float(line.split(":", 1)[1])
    t = vals.get("traffic_bytes_per_launch:")
    if t is None:
        return None
    if rows is not None and vals.get("captured_rows:"):
        t *= rows / vals["captured_rows:"]
    return t


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples: list[list[str]] = []
        self._stop = threading.Event()
        self._t: threading.Thread | None = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def gen_scan_table(rows: int, seed: int) -> dict[str, np.ndarray]:
    from turbogp_b200 import datagen
    full = datagen.lineitem(0, seed)  # column names / dtypes
    out = {}
    for name in SCAN_COLUMNS:
        rng = datagen._rng(seed, name)
        lo_hi = {"quantity": (1, 51), "price_cents": (90_000, 10_500_001), "discount_pct": (0, 11),
                 "ship_day": (datagen.DAY0, datagen.DAY0 + datagen.NDAYS)}[name]
        out[name] = rng.integers(lo_hi[0], lo_hi[1], rows, dtype=full[name].dtype)
    return out


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


# ---------------------------------------------------------------------------
# Reference arm: the C++ restatements of the reference's CPU paths
# ---------------------------------------------------------------------------
def cpu_workload_runner(name: str, n: int, threads: int):
    """(run(m) -> seconds of one pass over the first m rows, sample cap,
    description of what is timed) for a workload's reference CPU path."""
    from oracle import refpath
    from turbogp_b200 import datagen, workloads
    CT = datagen.LINEITEM_COLTYPES
    if name == "filtered_group_agg":
        cap = n
        tpl = workloads.filtered_group_agg()
        host = datagen.lineitem(cap, seed=1)
        run = lambda m: refpath.grouped_q1({k: v[:m] for k, v in host.items()}, tpl, CT, threads=threads)["seconds"]
        how = (f"rows of the same lineitem distributions through the C++ restatement of the reference's grouped "
               f"path (execute_grouped: 65,536-row chunks grouped on {threads} threads, per-group i64 / f64 sums)")
    elif name == "join_group_agg":
        cap = min(n, 20_000_000)
        tpl = workloads.join_group_agg()
        dim = datagen.dimension(DIM_ROWS, seed=2)
        fact_full = datagen.fact_fk(cap, DIM_ROWS, 0.8, seed=3)
        fact = {k: fact_full[k] for k in ("fk", "price_cents", "discount_pct")}
        del fact_full
        day_lt = tpl.build_where.ops[0][3]
        run = lambda m: refpath.join_group({k: v[:m] for k, v in fact.items()}, dim, day_lt, threads=threads)["seconds"]
        how = (f"probe rows (Zipf(0.8) fk over the 1.5M-row dimension, which is joined whole) through the C++ "
               f"restatement of the reference's join path (hash_join_with_keys: CRC32-tagged chained table + bloom "
               f"filter, 65,536-row probe chunks on {threads} threads, materialised join, then execute_grouped)")
    else:
        cap = min(n, 20_000_000)
        host = datagen.highcard(cap, 10_000_000, 1.1, seed=4)
        run = lambda m: refpath.highcard({k: v[:m] for k, v in host.items()}, threads=threads, cap=0)["seconds"]
        how = (f"rows of the same Zipf(1.1) key distribution through the C++ restatement of the reference's "
               f"accumulator grouping (try_accumulator_grouped: 65,536-row chunks into per-chunk hash maps on "
               f"{threads} threads, merged into one map)")
    return run, cap, how


def time_cpu_workload(name: str, n: int, warmup: int, steps: int, budget_s: float) -> dict:
    """Bounded-sample timing of a workload's reference CPU path: each step is
    one pass over the first `rows` rows, sized so warmup + steps take about
    budget_s seconds."""
    threads = os.cpu_count() or 1
    run, cap, how = cpu_workload_runner(name, n, threads)
    probe = min(cap, 100_000)
    per_row = run(probe) / probe
    rows = int(max(min(cap, 100_000), min(cap, budget_s / (warmup + steps) / max(per_row, 1e-12))))
    times = []
    for i in range(warmup + steps):
        t = run(rows)
        if i >= warmup:
            times.append(t)
    sec = sum(times)
    value = rows * len(times) / sec
    return {"value": value, "unit": "rows/s", "cores": threads, "kind": "port", "rows": rows,
            "ms_per_step": 1000 * sec / len(times), "sample": f"{rows} {how} per step"}


def reference_line(args, world: int, name: str, n: int, cpu: dict, config: dict) -> dict:
    return {
        "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": DATA,
        "config": config,
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cpu["value"], "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, world: int, rank: int) -> None:
    """The reference arm: the C++ restatement of the reference's CPU path for
    the scan (single-threaded, as the reference's interpreter runs that query),
    each step a bounded sample of the 60M rows; at the default workload the
    line also carries the other workloads' reference CPU paths, on all host
    threads, as `workloads`."""
    if rank != 0:
        return
    from oracle import refpath
    from turbogp_b200 import workloads
    tpl = workloads.selective_scan_sum()
    full = gen_scan_table(args.reference_rows, seed=1)
    threads = os.cpu_count() or 1
    # Each step is a bounded sample of the workload: one timed full pass sizes
    # it so the whole --warmup + --steps run is about a minute of CPU work.
    t_full = refpath.selective_scan_sum(full, tpl, threads=threads)["seconds"]
    budget_s = 60.0
    rows = int(min(args.reference_rows,
                   max(1_000_000, args.reference_rows * (budget_s / (args.warmup + args.steps)) / max(t_full, 1e-6))))
    cols = {k: v[:rows] for k, v in full.items()}
    times = []
    r = None
    for i in range(args.warmup + args.steps):
        r = refpath.selective_scan_sum(cols, tpl, threads=threads)
        if i >= args.warmup:
            times.append(r["seconds"])
    sec = sum(times)
    value = rows * len(times) / sec
    cpu = {"value": value, "unit": "rows/s", "cores": r["threads"], "kind": "port",
           "ms_per_step": 1000 * sec / len(times),
           "sample": f"first {rows} of the {args.reference_rows} rows per step, C++ restatement of the reference "
                     f"CPU path (single-threaded, as the reference runs this query)"}
    line = reference_line(args, world, "selective_scan_sum", args.reference_rows, cpu,
                          headline_config(world, args.reference_rows))
    if not args.no_workloads and args.reference_rows == ROWS:
        recs = {}
        for name, n in FULL_ROWS.items():
            c = time_cpu_workload(name, n, 1, 3, budget_s=12.0)
            recs[name] = {"value": c["value"], "unit": "rows/s", "ms_per_step": c["ms_per_step"],
                          "config": workload_config(name, n),
                          "cpu_baseline": {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")},
                          "e2e": {"value": c["value"], "unit": "rows/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}
        recs["batch"] = {"unavailable": "the reference has no batched-submission CPU path (its interpreter runs "
                                        "one statement at a time)"}
        line["workloads"] = recs
    print(json.dumps(line), flush=True)


def run_reference_workload(args, world: int, rank: int) -> None:
    """Reference arm of one grouped / join / high-cardinality workload (rank 0
    alone). The batch and serving workloads have no CPU counterpart in the
    reference (its server runs one statement at a time): they print the
    unavailable line."""
    if rank != 0:
        return
    name = args.workload
    if name in ("batch", "serve", "pgwire", "merged"):
        print(json.dumps({"impl": "reference", "unavailable": f"{name}: the reference has no batched-submission "
                          "or serving CPU path to time (the plain one-query-at-a-time arm is in this "
                          "workload's own line)"}), flush=True)
        return
    n = args.rows if args.rows != ROWS else FULL_ROWS[name]
    cpu = time_cpu_workload(name, n, args.warmup, args.steps, budget_s=60.0)
    print(json.dumps(reference_line(args, world, name, n, cpu, workload_config(name, n))), flush=True)


# ---------------------------------------------------------------------------
# The GPU arm of the grouped / join / high-cardinality / batch workloads
# ---------------------------------------------------------------------------
def same_output(a, b) -> bool:
    if a.rows_selected != b.rows_selected or a.keys != b.keys or len(a.values) != len(b.values):
        return False
    for ra, rb in zip(a.values, b.values):
        for x, y in zip(ra, rb):
            if x.count != y.count or x.value != y.value:
                return False
            if not (x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)):
                return False
    return True


def result_summary(out, limit: int = 6) -> list:
    """The first groups of a result as [key..., value...] lists (JSON-safe)."""
    rows = []
    for k, vals in list(zip(out.keys, out.values))[:limit]:
        rows.append([*k, *[str(v.value) for v in vals]])
    return rows


def measure_workload(name: str, ctx, args, world: int, rank: int, local: int, shared: dict | None = None) -> dict:
    """One workload at full size: timed steps (device events), the dominant
    kernel's gated launch time (roofline), the end-to-end step from pinned
    host buffers, and the CPU leg (reference CPU path on a bounded sample, and
    the exact check of the GPU's first result). Returns the record."""
    import torch
    from turbogp_b200 import datagen, workloads
    from turbogp_b200.engine import col, count_star, sum_
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    CT = datagen.LINEITEM_COLTYPES
    shared = shared if shared is not None else {}
    probe_only = None  # (callable, algorithmic bytes per launch) when the step has several kernels
    variant = None     # (description, callable): the same query with ORDER BY ... LIMIT, timed beside it
    n = args.rows if (args.rows != ROWS and args.workload == name) else FULL_ROWS[name]
    if name == "filtered_group_agg":
        tpl = workloads.filtered_group_agg()
        host = datagen.lineitem(n, seed=1 + rank)
        t = ctx.register(host, CT)
        q = t.prepare(tpl.aggs, tpl.group_by, tpl.where)
        step = q.run
        tables = [(t, host)]
        kernel_bytes = 26 * n
        dominant = "q1_group_kernel (streaming loads, per-thread private partials, 6 direct groups)"
        traffic = traffic_per_launch("filtered_group_agg_6M_q1_group_kernel.md", n)
        check = lambda out: _check_exact(out, host, CT, tpl.aggs, tpl.group_by, tpl.where)
        cleanup = [t.drop]
    elif name == "join_group_agg":
        tpl = workloads.join_group_agg()
        dim = datagen.dimension(DIM_ROWS, seed=2 + rank)
        fact_full = shared.get("fact") if shared.get("fact") is not None and rank == 0 else \
            datagen.fact_fk(n, DIM_ROWS, 0.8, seed=3 + rank)
        fact = {k: np.ascontiguousarray(fact_full[k][:n]) for k in ("fk", "price_cents", "discount_pct")}
        fct = {"fk": "int", "price_cents": "int", "discount_pct": "int"}
        d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
        f = ctx.register(fact, fct)

        def step():
            j = d.join_build("key", tpl.build_where)
            out = f.aggregate(tpl.aggs, tpl.group_by, tpl.where, join=j, probe_key="fk")
            j.drop()
            return out

        j0 = d.join_build("key", tpl.build_where)
        pq = f.prepare(tpl.aggs, tpl.group_by, tpl.where, join=j0, probe_key="fk")
        q = pq
        probe_only = (pq.run, 16 * n, pq)
        tables = [(d, dim), (f, fact)]
        kernel_bytes = 16 * n
        dominant = "scan_kernel<MODE_GROUP_SHARED32, 512, DenseShape<join>, 2 CTAs per SM> join probe + GROUP BY segment (25 groups, payload array)"
        traffic = traffic_per_launch("join_group_agg_probe_kernel.md", n)
        build = (dim, datagen.DIMENSION_COLTYPES, "key", tpl.build_where)
        check = lambda out: _check_exact(out, fact, fct, tpl.aggs, tpl.group_by, tpl.where, build, "fk")
        cleanup = [j0.drop, f.drop, d.drop]
    else:  # highcard_group
        host = shared.get("hc") if shared.get("hc") is not None and rank == 0 else \
            datagen.highcard(n, 10_000_000, 1.1, seed=4 + rank)
        t = ctx.register(host)
        aggs = [count_star(), sum_(col("value"))]
        q = t.prepare(aggs, ("key",), None, group_cap=10_000_000)
        step = lambda: q.run(decode=False)
        variant = ("ORDER BY count(*) DESC LIMIT 10 (tgp_execute_topn)",
                   lambda: t.aggregate_topn(aggs, ("key",), None, 0, True, 10))
        tables = [(t, host)]
        kernel_bytes = 12 * n
        dominant = "direct_group_kernel<int64 key, int32 value> (one-word direct slots, shared table of hot keys)"
        traffic = traffic_per_launch("highcard_group_direct_group_kernel.md", n)
        check = lambda out: _check_highcard(q, host)
        cleanup = [t.drop]

    first = step() if name != "highcard_group" else q.run()
    # The autotuner measures the dominant scan's variants (each checked
    # against the planner's result bit for bit) and installs the fastest for
    # this query class; the timed steps below run it.
    tune = None if args.no_autotune else autotune_summary(ctx, probe_only[2] if probe_only is not None else q)
    for _ in range(args.warmup):
        step()
    steps = args.steps if args.steps != 3000 else 20
    ctx.profile(True)
    ctx.profile_read()
    torch.cuda.synchronize()
    ctx.sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
    launches, _ = ctx.profile_read()
    ms = ev0.elapsed_time(ev1)
    # Kernel time alone: each launch queued behind a short device delay.
    ctx.profile(True, gated=True)
    run_one = probe_only[0] if probe_only is not None else step
    for _ in range(3):
        run_one()
    ctx.profile_read()
    for _ in range(steps):
        run_one()
    pl, pms = ctx.profile_read()
    kernel_avg = pms / max(1, pl)
    ctx.profile(False)

    # e2e: pinned host buffers re-uploaded every step, result read back.
    pinned = [(tb, {k: torch.from_numpy(v).pin_memory().numpy() for k, v in h.items()}) for tb, h in tables]
    h2d = sum(a.nbytes for _, h in pinned for a in h.values())
    e2e_steps = max(1, min(args.e2e_steps, 5))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        for tb, h in pinned:
            tb.reload(h)
        out = step()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    ngroups = int(q.res.ngroups)
    nk, na = q.nk, q.na
    d2h = ngroups * (8 * nk + 32 * na) + 48   # keys, one 32-byte value record per aggregate, counters
    del pinned

    variant_line = None
    if variant is not None:
        for _ in range(2):
            variant[1]()
        v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        v0.record(stream)
        for _ in range(steps):
            variant[1]()
        v1.record(stream)
        v1.synchronize()
        variant_line = {"query": variant[0], "ms_per_step": v0.elapsed_time(v1) / steps}

    # CPU leg (rank 0 at N=1): the exact check of the first result, then the
    # reference's CPU path on a bounded sample.
    cpu, checked = None, None
    if rank == 0 and world == 1:
        checked = check(first)
        if not checked["ok"]:
            raise SystemExit(f"{name}: GPU result differs from the exact checker: {checked}")
        if not args.no_cpu_baseline:
            c = time_cpu_workload(name, n, 1, 2, budget_s=8.0)
            cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
    for fn in cleanup:
        fn()
    rows_step = n + (DIM_ROWS if name == "join_group_agg" else 0)
    bytes_step = workload_config(name, n)["bytes_per_step"]
    peak, peak_kind = peak_hbm()
    achieved = kernel_bytes / (kernel_avg / 1000.0) / 1e9
    rec = {
        "metric": METRIC, "value": rows_step * world * steps / (ms / 1000.0), "unit": "rows/s", "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": DATA,
        "config": workload_config(name, n),
        "hbm_gbs": bytes_step * world * steps / (ms / 1000.0) / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic, "kernel_ms": kernel_avg, "kernel": dominant,
                     "timing": "device events around each launch, launch queued behind a device delay"},
        "e2e": {"value": rows_step * e2e_steps / (e2e_ms / 1000.0), "unit": "rows/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "cpu_baseline": cpu, "clocks": clocks.summary(), "gpu_launches": launches,
        "result": checked,
    }
    if variant_line is not None:
        rec["variant"] = variant_line
    rec["autotune"] = tune
    return rec


def autotune_summary(ctx, pq, reps: int = 5) -> dict:
    """tgp_autotune on a prepared query: the planner's rule against the
    fastest candidate (both gated CUDA-event medians of the scan kernel)."""
    rep = ctx.autotune(pq, reps=reps)
    cands = rep["candidates"]
    best = cands[rep["best"]]
    return {"rule_ms": rep["rule_ms"], "best_ms": rep["best_ms"], "chosen": best["variant"],
            "chosen_placement": best["mode"], "chosen_threads": best["threads"], "chosen_stages": best["stages"],
            "rule_placement": cands[0]["mode"], "candidates": len(cands),
            "all_same_result": all(c["same_result"] for c in cands if c["status"] == 0)}


def _check_exact(out, cols, coltypes, aggs, group_by, where, build=None, probe_key=None) -> dict:
    """The GPU result against the exact numpy checker (oracle/scale.py)."""
    from oracle import scale
    exp = scale.aggregate(cols, coltypes, aggs, group_by, where, build=build, probe_key=probe_key)
    return {"ok": same_output(out, exp), "checker": "oracle.scale.aggregate (exact)", "groups": len(out.keys),
            "rows_selected": out.rows_selected, "first_groups": result_summary(out)}


def _check_highcard(q, host) -> dict:
    """Every group of the GROUP BY key result against numpy bincounts."""
    from oracle import scale
    keys, lo, hi, cnt = q._output(q.res).arrays()
    ek, ec, es = scale.group_count_sum(host["key"], host["value"])
    ok = (keys.shape[0] == ek.shape[0] and np.array_equal(keys[:, 0], ek) and
          np.array_equal(lo[:, 0].view(np.int64), ec) and np.array_equal(lo[:, 1].view(np.int64), es) and
          not hi.any())
    return {"ok": bool(ok), "checker": "oracle.scale.group_count_sum (exact bincounts)", "groups": int(keys.shape[0]),
            "rows_selected": int(q.res.rows_selected)}


def batch_queries(ctx, fact_dev: dict, dim_host: dict, nq: int, seed: int):
    """The batching workload's queries: nq prepared queries, each over a prefix
    view of the resident 60M-row fact table whose size is log-uniform in
    [10K, 60M] rows, with a template drawn from (selective scan + sum,
    filtered grouped aggregate, join + grouped aggregate) and random literals
    (selectivity about 0.1% to 90%). Views share the device columns."""
    import numpy as np
    from turbogp_b200 import datagen, workloads
    from turbogp_b200.engine import col
    rng = np.random.default_rng(seed)
    d = ctx.register(dim_host, datagen.DIMENSION_COLTYPES)
    tj = workloads.join_group_agg()
    j = d.join_build("key", tj.build_where)
    fct = {**datagen.LINEITEM_COLTYPES, "fk": "int"}
    n_all = next(iter(fact_dev.values())).numel()
    views, pqs, rows, nbytes = {}, [], [], []
    for _ in range(nq):
        n = int(min(n_all, round(float(np.exp(rng.uniform(np.log(1e4), np.log(6e7)))))))
        if n not in views:
            views[n] = ctx.register_device({k: v[:n] for k, v in fact_dev.items()}, fct)
        t = views[n]
        kind = int(rng.integers(0, 3))
        if kind == 0:
            tpl = workloads.selective_scan_sum(day_lo=datagen.DAY0 + int(rng.integers(0, 2000)),
                                               days=int(rng.integers(30, 526)), disc_lo=int(rng.integers(0, 6)),
                                               disc_hi=int(rng.integers(5, 11)), qty_lt=int(rng.integers(2, 51)))
            pqs.append(t.prepare(tpl.aggs, tpl.group_by, tpl.where))
            nbytes.append(20 * n)   # ship_day, discount_pct, quantity, price_cents
        elif kind == 1:
            tpl = workloads.filtered_group_agg(ship_max=datagen.DAY0 + int(rng.integers(3, datagen.NDAYS)))
            pqs.append(t.prepare(tpl.aggs, tpl.group_by, tpl.where))
            nbytes.append(26 * n)   # the seven lineitem columns
        else:
            pqs.append(t.prepare(tj.aggs, tj.group_by, col("quantity") < int(rng.integers(2, 51)), join=j,
                                 probe_key="fk"))
            nbytes.append(20 * n)   # fk, price_cents, discount_pct, quantity
        rows.append(n)
    return pqs, rows, nbytes, (d, j, views)


def measure_batch(ctx, args, world: int, rank: int, local: int, fact_host: dict | None = None) -> dict:
    """Batching: 256 queries of uneven sizes (see batch_queries) per step, run
    as one tgp_batch_submit (persistent launch over a device morsel queue)
    against the same 256 queries issued one by one (plan, launch, readback
    per query). value = batched queries/s; plain_qps beside it. The CPU leg
    checks every batched result against the same query run alone, and the
    smallest and largest query of each template against the exact checker."""
    import torch
    from turbogp_b200 import datagen, workloads
    nq = 256
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    n = args.rows if (args.rows != ROWS and args.workload == "batch") else 60_000_000
    host = fact_host if fact_host is not None and rank == 0 else datagen.fact_fk(n, DIM_ROWS, 0.8, seed=3 + rank)
    fact = {k: torch.from_numpy(v[:n]).to(f"cuda:{local}") for k, v in host.items()}
    dim = datagen.dimension(DIM_ROWS, seed=2 + rank)
    pqs, rows, nbytes, keep = batch_queries(ctx, fact, dim, nq, seed=11 + rank)
    total_rows = sum(rows)
    steps = args.steps if args.steps != 3000 else 5

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    first_batched = ctx.submit(pqs).wait()
    first_plain = [q.run() for q in pqs]
    batch = lambda: ctx.submit(pqs, decode=False).wait()
    plain = lambda: [q.run(decode=False) for q in pqs]
    for _ in range(args.warmup):
        batch()
    plain()
    ctx.profile(True)
    ctx.profile_read()
    with ClockSampler(local) as clocks:
        ms_batch = timed(batch, steps)
    launches, kern_ms = ctx.profile_read()
    k_plain = max(1, steps // 2)
    ms_plain = timed(plain, k_plain) / k_plain * steps
    ctx.profile(False)
    # e2e: results read back into host buffers by every query of the batch
    # (the tables stay resident, as they do for a served query).
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.submit(pqs, decode=True).wait()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    d2h = sum(int(q.res.ngroups) * (8 * q.nk + 32 * q.na) + 48 for q in pqs)
    checked = None
    if rank == 0 and world == 1:
        from oracle import scale
        same = all(same_output(b, p) for b, p in zip(first_batched, first_plain))
        tj = workloads.join_group_agg()
        build = (dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
        fct = {**datagen.LINEITEM_COLTYPES, "fk": "int"}
        picked = {}
        for i, pq in enumerate(pqs):
            shape = (pq.nk, pq.na, int(pq.q.join != 0))
            lo, hi = picked.get(shape, (i, i))
            picked[shape] = (lo if rows[lo] <= rows[i] else i, hi if rows[hi] >= rows[i] else i)
        exact = True
        sample = sorted({i for pair in picked.values() for i in pair})
        for i in sample:
            sp = pqs[i].spec
            view = {k: v[:rows[i]] for k, v in host.items()}
            e = scale.aggregate(view, fct, sp["aggs"], sp["group_by"], sp["where"],
                                build=build if sp["join"] is not None else None,
                                probe_key="fk" if sp["join"] is not None else None)
            exact = exact and same_output(first_batched[i], e)
        checked = {"ok": bool(same and exact), "checker": "every batched result == the query run alone; "
                   f"{len(sample)} of them (smallest and largest of each template) == oracle.scale.aggregate",
                   "queries": nq}
        if not checked["ok"]:
            raise SystemExit(f"batch: results differ: {checked}")
    peak, peak_kind = peak_hbm()
    achieved = sum(nbytes) / (kern_ms / steps / 1000.0) / 1e9 if kern_ms else None
    rec = {
        "metric": METRIC, "value": nq * world * steps / (ms_batch / 1000.0), "unit": "queries/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": ms_batch / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": DATA,
        "config": {"workload": f"batch of {nq} queries (sizes log-uniform 10K-60M rows over prefix views of a "
                               f"{n}-row resident table; selective scan+sum / filtered grouped aggregate / "
                               f"join+grouped aggregate with random literals) per step",
                   "rows_per_step": total_rows, "l2": "inputs larger than the 126 MB L2"},
        "plain_qps": nq * steps / (ms_plain / 1000.0), "ms_plain_per_step": ms_plain / steps,
        "rows_per_s": total_rows * steps / (ms_batch / 1000.0),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "peak_kind": peak_kind, "traffic": None,
                     "kernel_ms_per_step": kern_ms / steps, "kernel": "batch_kernel (persistent, device morsel queue)",
                     "timing": "summed device events around the batch's launches"},
        "e2e": {"value": nq * steps / (e2e_ms / 1000.0), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": d2h,
                "note": "tables resident in HBM (served-query setting); every result decoded on the host"},
        "cpu_baseline": None, "clocks": clocks.summary(), "gpu_launches": launches, "result": checked,
    }
    d, j, views = keep
    j.drop()
    for v in views.values():
        v.drop()
    d.drop()
    return rec


def run_workload(args, world: int, rank: int, local: int) -> None:
    """One JSON line for one non-headline workload (--workload NAME)."""
    from turbogp_b200.engine import Context
    ctx = Context(local)
    if args.workload == "batch":
        rec = measure_batch(ctx, args, world, rank, local)
    elif args.workload == "merged":
        rec = measure_merged(ctx, args, world, rank, local)
    else:
        rec = measure_workload(args.workload, ctx, args, world, rank, local)
    if rank == 0:
        print(json.dumps(rec), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def serve_templates(f, j):
    """The three light serving templates over the fact table (and the join)."""
    from turbogp_b200 import workloads
    t_scan, t_fga, tj = workloads.selective_scan_sum(), workloads.filtered_group_agg(), workloads.join_group_agg()
    return {"scan": lambda: f.prepare(t_scan.aggs, t_scan.group_by, t_scan.where),
            "fga": lambda: f.prepare(t_fga.aggs, t_fga.group_by, t_fga.where),
            "join": lambda: f.prepare(tj.aggs, tj.group_by, None, join=j, probe_key="fk")}


def serve_literals(rng, kind):
    """A request's WHERE for a light serving template, random literals."""
    from turbogp_b200 import datagen
    from turbogp_b200.engine import col
    D0, ND = datagen.DAY0, datagen.NDAYS
    if kind == "scan":
        lo = D0 + int(rng.integers(0, ND - 30))
        return ((col("ship_day") >= lo) & (col("ship_day") < lo + int(rng.integers(30, 366))) &
                col("discount_pct").between(int(rng.integers(0, 6)), int(rng.integers(5, 11))) &
                (col("quantity") < int(rng.integers(2, 51))))
    if kind == "fga":
        return col("ship_day") <= D0 + int(rng.integers(3, ND))
    return col("quantity") < int(rng.integers(2, 51))


def measure_merged(ctx, args, world: int, rank: int, local: int, fact_host: dict | None = None) -> dict:
    """Merged scans: per light serving template, a batch of `--members`
    requests with random literals (one merged scan per template class, plus a
    per-bucket count scan for the join) against one of them run alone. Device
    time from events around each scan launch (queued behind a device delay);
    every member of the first batch is checked against the same request run
    alone. With --profile-window, the timed batches run between
    cudaProfilerStart and cudaProfilerStop (for `ncu --profile-from-start off`)."""
    import numpy as np
    import torch
    from turbogp_b200 import datagen, workloads
    n = args.rows if (args.rows != ROWS and args.workload == "merged") else 60_000_000
    host = fact_host if fact_host is not None and rank == 0 else datagen.fact_fk(n, DIM_ROWS, 0.8, seed=3 + rank)
    f = ctx.register({k: v[:n] for k, v in host.items()}, {**datagen.LINEITEM_COLTYPES, "fk": "int"})
    d = ctx.register(datagen.dimension(DIM_ROWS, seed=2 + rank), datagen.DIMENSION_COLTYPES)
    j = d.join_build("key", workloads.join_group_agg().build_where)
    make = serve_templates(f, j)
    kinds = [args.merged_class] if args.merged_class else list(make)
    rng = np.random.default_rng(31 + rank)
    nb = args.members
    steps = args.steps if args.steps != 3000 else 5
    out = {}
    for kind in kinds:
        pqs = [make[kind]() for _ in range(nb)]
        batch = [pq.rebind(serve_literals(rng, kind)) for pq in pqs]
        merged = ctx.submit(batch).wait()
        alone = [make[kind]().rebind(pq.spec["where"]).run() for pq in batch]
        same = all(same_output(a, b) for a, b in zip(merged, alone))
        if not same:
            raise SystemExit(f"merged {kind}: a member differs from the same request alone")
        for _ in range(args.warmup):
            ctx.submit([pq.rebind(serve_literals(rng, kind)) for pq in pqs], decode=False).wait()
        ctx.profile(True, gated=True)
        ctx.profile_read()
        if args.profile_window:
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStart()
        per = []
        for _ in range(steps):
            ctx.submit([pq.rebind(serve_literals(rng, kind)) for pq in pqs], decode=False).wait()
            per.append(ctx.profile_read())
        if args.profile_window:
            torch.cuda.cudart().cudaProfilerStop()
        one = make[kind]()
        plain = []
        for _ in range(steps):
            one.rebind(serve_literals(rng, kind)).run(decode=False)
            plain.append(ctx.profile_read()[1])
        ctx.profile(False)
        mk = float(np.median([ms for _, ms in per]))
        pk = float(np.median(plain))
        out[kind] = {"members": nb, "merged_kernel_ms": mk, "launches": int(per[0][0]), "alone_kernel_ms": pk,
                     "alone_ms_x_members_over_merged": pk * nb / mk if mk else None, "same_as_alone": same}
    j.drop()
    f.drop()
    d.drop()
    return {"workload": f"merged scans: {nb} requests of each light serving template with random literals over "
                        f"a {n}-row fact table, one batch", "records": out, "steps": steps,
            "timing": "device events around each scan launch, launch queued behind a device delay"}


def measure_serve(ctx, args, world: int, rank: int, local: int, fact_host: dict | None = None,
                  hc_host: dict | None = None) -> dict:
    """Serving: resident 60M-row fact table, 1.5M-row dimension (+ join table)
    and a 100M-row high-cardinality table; open-loop Poisson streams of
    requests (selective scan + sum, filtered grouped aggregate, join + grouped
    aggregate, each with random literals; GROUP BY key over the
    high-cardinality table for 1 in 500) served by the continuous-batching
    server (merged and shared scans, planner-sized admission, a heavy lane on
    its own context) and by plain one-at-a-time execution.

    Measured: the plain server's capacity (completed q/s with arrivals far
    above it) and its p50 / p99 at 80 % of that capacity; the batched server's
    policy (batches in flight: 1 or 2) picked on a calibration stream at 5x
    the plain capacity; then the batched server offered 5x, 6x, 8x, 10x, 12x,
    14x, 16x the plain capacity, until its p99 exceeds the plain p99 or it
    falls behind the offered rate; and its own capacity. value = the highest
    completed q/s whose p99 is at most the plain server's p99 (the 5x run's,
    if none is)."""
    import numpy as np
    from turbogp_b200 import datagen, serving, workloads
    from turbogp_b200.engine import Context, col, count_star, sum_
    n = args.rows if (args.rows != ROWS and args.workload == "serve") else 60_000_000
    host = fact_host if fact_host is not None and rank == 0 else datagen.fact_fk(n, DIM_ROWS, 0.8, seed=3 + rank)
    f = ctx.register({k: v[:n] for k, v in host.items()}, {**datagen.LINEITEM_COLTYPES, "fk": "int"})
    d = ctx.register(datagen.dimension(DIM_ROWS, seed=2 + rank), datagen.DIMENSION_COLTYPES)
    tj = workloads.join_group_agg()
    j = d.join_build("key", tj.build_where)
    # The high-cardinality table lives on a second context (its own stream):
    # the batched server runs its requests in a heavy lane beside the batches.
    ctx_heavy = Context(local)
    hch = hc_host if hc_host is not None and rank == 0 else \
        datagen.highcard(args.highcard_rows, 10_000_000, 1.1, seed=4 + rank)
    hc = ctx_heavy.register(hch)
    hc_aggs = [count_star(), sum_(col("value"))]
    templates = {name: serving.Template(name, mk) for name, mk in serve_templates(f, j).items()}
    templates["highcard"] = serving.Template("highcard", lambda: hc.prepare(hc_aggs, ("key",), None,
                                                                            group_cap=10_000_000), heavy=True)
    rng = np.random.default_rng(21 + rank)

    def request(t):
        u = rng.random()
        if u < 0.002:
            return serving.Request(t, "highcard", None)
        kind = ("scan", "fga", "join")[int(rng.integers(0, 3))]
        return serving.Request(t, kind, serve_literals(rng, kind))

    def stream(rate, count):
        return [request(t) for t in serving.poisson_arrivals(rate, count, rng)]

    count = args.requests
    # Warm-up: every template's prepared queries built and sized (the
    # high-cardinality one included), then both paths once.
    serving.prewarm(templates, [request(0.0) for _ in range(2000)], per_template=4)
    serving.reserve(templates, 640)   # two full batches of one template in flight and queued
    serving.serve_batched(ctx, templates, stream(4000.0, 256), mem_budget=args.mem_budget)
    serving.serve_plain(ctx, templates, stream(4000.0, 32))
    # Plain capacity, then plain at 80 % of it.
    plain_sat = serving.serve_plain(ctx, templates, stream(50_000.0, max(400, count // 4)))
    cap_p = plain_sat["qps"]
    plain = serving.serve_plain(ctx, templates, stream(0.8 * cap_p, max(400, count // 2)))
    p99_plain = plain.get("p99_ms") or 0.0
    # Policy: batches in flight, on a calibration stream of its own.
    calib = {}
    for inflight in (1, 2):
        r = serving.serve_batched(ctx, templates, stream(5.0 * cap_p, max(600, count // 2)),
                                  mem_budget=args.mem_budget, max_inflight=inflight)
        calib[inflight] = r.get("p99_ms") or 1e9
    inflight = min(calib, key=calib.get)
    ladder, best = [], None
    with ClockSampler(local) as clocks:
        for m in (5.0, 6.0, 8.0, 10.0, 12.0, 14.0, 16.0):
            r = serving.serve_batched(ctx, templates, stream(m * cap_p, count), mem_budget=args.mem_budget,
                                      max_inflight=inflight)
            r = {**r, "offered_qps": m * cap_p, "offered_x_plain_capacity": m}
            ladder.append(r)
            ok = (r.get("p99_ms") or 1e9) <= p99_plain
            if ok:
                best = r
            # (A stream's completed q/s sits a few percent under its offered
            # rate: the window ends with the last completion, which can be a
            # high-cardinality request of several ms.)
            if not ok or (r.get("qps") or 0) < 0.85 * m * cap_p:
                break
    batched_sat = serving.serve_batched(ctx, templates, stream(100_000.0, count), mem_budget=args.mem_budget,
                                        max_inflight=inflight)
    at5 = ladder[0]
    head = best if best is not None else at5
    rec = {
        "metric": METRIC, "value": head.get("qps"), "unit": "queries/s", "n_gpus": world,
        "steps": count, "warmup": 256, "ms_per_step": head.get("mean_ms"), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": DATA,
        "config": {"workload": f"serving: Poisson arrivals of scan+sum / filtered grouped aggregate / join+grouped "
                               f"aggregate over a resident {n}-row fact table (random literals) and GROUP BY key "
                               f"over a {args.highcard_rows}-row high-cardinality table (1 in 500); continuous "
                               f"batching with merged and shared scans, planner-sized admission (budget "
                               f"{args.mem_budget} B), high-cardinality requests in a heavy lane (own stream)",
                   "requests": count, "value": "highest batched completed q/s with p99 <= the plain p99 at 80% "
                                               "of plain capacity" if best is not None else
                                               "batched completed q/s at 5x plain capacity (p99 above plain)"},
        "plain_capacity_qps": cap_p,
        "plain_at_80pct": {**plain, "offered_qps": 0.8 * cap_p},
        "batched_policy": {"max_inflight": inflight, "calibration_p99_ms": calib},
        "batched_at_5x": at5,
        "batched_ladder": ladder,
        "batched_capacity_qps": batched_sat.get("qps"),
        "qps_ratio_at_5x": (at5.get("qps") or 0) / cap_p if cap_p else None,
        "p99_batched_le_plain": (at5.get("p99_ms") or 1e9) <= p99_plain,
        "batched_qps_at_plain_p99": best.get("qps") if best is not None else None,
        "ratio_at_plain_p99_vs_plain_capacity": (best.get("qps") / cap_p) if best is not None and cap_p else None,
        "ratio_at_plain_p99_vs_plain_at_80pct": (best.get("qps") / plain["qps"]) if best is not None and
                                                plain.get("qps") else None,
        "roofline": None, "e2e": None, "cpu_baseline": None, "clocks": clocks.summary(), "gpu_launches": None,
    }
    j.drop()
    for tpl in templates.values():
        tpl.pool.clear()
    hc.drop()
    ctx_heavy.close()
    f.drop()
    d.drop()
    return rec


def run_serve(args, world: int, rank: int, local: int) -> None:
    from turbogp_b200.engine import Context
    ctx = Context(local)
    rec = measure_serve(ctx, args, world, rank, local)
    if rank == 0:
        print(json.dumps(rec), flush=True)
    ctx.close()


# ---------------------------------------------------------------------------
# Headline: the 60M-row selective scan
# ---------------------------------------------------------------------------
def run_headline(args, world: int, rank: int, local: int) -> None:
    import torch
    from turbogp_b200 import workloads
    from turbogp_b200.engine import Context

    rows = args.rows
    tpl = workloads.selective_scan_sum()
    host = gen_scan_table(rows, seed=1 + rank)
    ctx = Context(local)
    coltypes = {"ship_day": "date", "discount_pct": "int", "quantity": "int", "price_cents": "int"}
    table = ctx.register(host, coltypes)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))

    def merge(out):
        """Exact cross-rank merge of the partial int128 sum and count: one NCCL
        all-gather of three int64 words per rank (turbogp_b200.shard holds the
        general merge of grouped results)."""
        if world == 1:
            return out.values[0][0].value, out.values[0][1].value
        import torch.distributed as dist
        s, c = out.values[0][0].value, out.values[0][1].value
        lo = int(np.array([s & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64).view(np.int64)[0])
        mine = torch.tensor([lo, s >> 64, c], dtype=torch.int64, device="cuda")
        parts = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine)
        tot_s, tot_c = 0, 0
        for p in parts:
            lo, hi, cc = [int(x) for x in p.cpu()]
            tot_s += (hi << 64) | (lo & 0xFFFFFFFFFFFFFFFF)
            tot_c += cc
        return tot_s, tot_c

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    query = table.prepare(tpl.aggs, tpl.group_by, tpl.where)
    first = query.run()
    tune = None if args.no_autotune else autotune_summary(ctx, query)
    # Warm-up.
    for _ in range(args.warmup):
        out = query.run()
        merge(out)
    expect = merge(out)

    # ---- value: table resident in HBM -------------------------------------
    ctx.profile(True)
    ctx.profile_read()
    barrier()
    torch.cuda.synchronize()
    ctx.sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            out = query.run()
            got = merge(out)
        ev1.record(stream)
        ev1.synchronize()
    ctx.sync()
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    launches, kernel_ms = ctx.profile_read()
    ctx.profile(False)
    if got != expect:
        raise SystemExit(f"result changed between steps: {got} != {expect}")
    clk = clocks.summary()
    kernel_avg_ungated_ms = max_over_ranks(kernel_ms / max(1, launches))
    # Kernel time alone: device events around each launch, with the launch
    # queued behind a short device delay so the host's submission of it (the
    # GPU is idle between synchronous queries) is not counted.
    ctx.profile(True, gated=True)
    ctx.profile_read()
    for _ in range(min(args.steps, 200)):
        query.run(decode=False)
    glaunch, gms = ctx.profile_read()
    ctx.profile(False)
    kernel_avg_ms = max_over_ranks(gms / max(1, glaunch))
    value = rows * world * args.steps / (ms / 1000.0)

    # ---- e2e: pinned host buffers, H2D + execute + D2H every step ----------
    pinned = {k: torch.from_numpy(v).pin_memory() for k, v in host.items()}
    pinned_np = {k: v.numpy() for k, v in pinned.items()}
    h2d = sum(v.nbytes for v in pinned_np.values())
    d2h = 8 * 6  # accumulator words + counters read back per step
    table.reload(pinned_np)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        table.reload(pinned_np)
        out = query.run()
        got = merge(out)
    e1.record(stream)
    e1.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = rows * world * args.e2e_steps / (e2e_ms / 1000.0)
    if got != expect:
        raise SystemExit("e2e result differs")
    del pinned, pinned_np

    # ---- CPU leg (rank 0, N=1 only): exact check + reference CPU path ------
    cpu, checked = None, None
    if rank == 0 and world == 1:
        checked = _check_exact(first, host, coltypes, tpl.aggs, (), tpl.where)
        if not checked["ok"]:
            raise SystemExit(f"selective_scan_sum: GPU result differs from the exact checker: {checked}")
        if not args.no_cpu_baseline:
            from oracle import refpath
            sample = min(args.cpu_sample_rows, rows)
            r = refpath.selective_scan_sum({k: v[:sample] for k, v in host.items()}, tpl,
                                           threads=os.cpu_count() or 1)
            cpu = {"value": sample / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
                   "sample": f"first {sample} rows of the same table, one pass, C++ restatement of the "
                             f"reference CPU path (AVX-512 filters into bitmaps, set-bit collect, f64 sum)"}

    peak, peak_kind = peak_hbm()
    achieved = rows * BYTES_PER_ROW / (kernel_avg_ms / 1000.0) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": DATA,
        "config": headline_config(world, rows),
        "hbm_gbs": rows * world * BYTES_PER_ROW * args.steps / (ms / 1000.0) / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic_per_launch(),
                     "kernel_ms": kernel_avg_ms, "kernel_ms_ungated": kernel_avg_ungated_ms,
                     "timing": "device events around each launch, launch queued behind a device delay",
                     "kernel": "scan_kernel<MODE_GROUP_PRIVATE, int64, 512, ScalarTag>"},
        "e2e": {"value": e2e_value, "unit": "rows/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
        "result": {"sum": str(expect[0]), "count": expect[1], **({"check": checked} if checked else {})},
        "autotune": tune,
    }
    table.drop()
    del host
    # The other workloads at full size (N=1 only: under torchrun the line
    # stays the headline's weak-scaling measurement).
    if world == 1 and not args.no_workloads and rows == ROWS:
        from turbogp_b200 import datagen
        recs = {}
        fact = datagen.fact_fk(60_000_000, DIM_ROWS, 0.8, seed=3)
        hc = datagen.highcard(FULL_ROWS["highcard_group"], 10_000_000, 1.1, seed=4)
        shared = {"fact": fact, "hc": hc}
        for name in ("filtered_group_agg", "join_group_agg", "highcard_group"):
            recs[name] = measure_workload(name, ctx, args, world, rank, local, shared)
        recs["batch"] = measure_batch(ctx, args, world, rank, local, fact_host=fact)
        recs["serve"] = measure_serve(ctx, args, world, rank, local, fact_host=fact, hc_host=hc)
        line["workloads"] = recs
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--reference-rows", type=int, default=ROWS)
    ap.add_argument("--cpu-sample-rows", type=int, default=ROWS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="headline line only (no `workloads` records)")
    ap.add_argument("--no-autotune", action="store_true", help="run the planner's rules (profiling captures)")
    ap.add_argument("--workload", default="selective_scan_sum",
                    choices=["selective_scan_sum", "filtered_group_agg", "join_group_agg", "highcard_group", "batch",
                             "serve", "merged"])
    ap.add_argument("--members", type=int, default=16, help="merged: requests per batch")
    ap.add_argument("--merged-class", default="", choices=["", "scan", "fga", "join"], help="merged: one template only")
    ap.add_argument("--profile-window", action="store_true",
                    help="merged: timed batches between cudaProfilerStart / Stop")
    ap.add_argument("--rate", type=float, default=2000.0, help="(unused: serve offers multiples of the plain capacity)")
    ap.add_argument("--requests", type=int, default=6000, help="serve: requests in the batched streams")
    ap.add_argument("--mem-budget", type=int, default=8 << 30, help="serve: admission budget in bytes")
    ap.add_argument("--highcard-rows", type=int, default=100_000_000)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        if args.workload == "selective_scan_sum":
            run_reference(args, world, rank)
        else:
            run_reference_workload(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "serve":
        run_serve(args, world, rank, local)
        return
    if args.workload != "selective_scan_sum":
        run_workload(args, world, rank, local)
        return
    run_headline(args, world, rank, local)


if __name__ == "__main__":
    main()
