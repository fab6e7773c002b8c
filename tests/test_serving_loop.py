"""The serving loop's host logic on CPU, with fake prepared queries and
batches: every request completes after it arrives, admission keeps the
in-flight memory under the budget, heavy requests run in their own lane while
batches go on, and an error in the heavy lane reaches the caller."""
import threading
import time

import numpy as np
import pytest

from turbogp_b200 import serving


class FakePQ:
    def __init__(self, name, log, delay=0.0, fail=False):
        self.name, self.log, self.delay, self.fail = name, log, delay, fail
        self.where = None

    def rebind(self, where):
        self.where = where
        return self

    def run(self, decode=True):
        self.log.append(("run", self.name, threading.get_ident()))
        if self.fail:
            raise RuntimeError("heavy query failed")
        time.sleep(self.delay)


class FakeHandle:
    def __init__(self, pqs, finish_at):
        self.pqs, self.finish_at = pqs, finish_at

    def poll(self):
        return time.perf_counter() >= self.finish_at

    def wait(self):
        while not self.poll():
            time.sleep(1e-4)


class FakeCtx:
    def __init__(self, batch_seconds, templates):
        self.batch_seconds, self.templates = batch_seconds, templates
        self.submitted, self.max_used = [], 0
        self.inflight: list[FakeHandle] = []

    def submit(self, pqs, decode=True):
        self.inflight = [h for h in self.inflight if not h.poll()]
        used = sum(self.templates[p.name].mem_bytes for h in self.inflight for p in h.pqs)
        used += sum(self.templates[p.name].mem_bytes for p in pqs)
        self.max_used = max(self.max_used, used)
        h = FakeHandle(list(pqs), time.perf_counter() + self.batch_seconds)
        self.inflight.append(h)
        self.submitted.append([p.name for p in pqs])
        return h


def make_templates(log, heavy_delay=0.05, heavy_fail=False):
    return {
        "light": serving.Template("light", lambda: FakePQ("light", log), 100),
        "big": serving.Template("big", lambda: FakePQ("big", log), 600),
        "heavy": serving.Template("heavy", lambda: FakePQ("heavy", log, heavy_delay, heavy_fail), 10**9,
                                  heavy=True),
    }


def requests(n, rate, seed, heavy_every=50):
    rng = np.random.default_rng(seed)
    arr = serving.poisson_arrivals(rate, n, rng)
    out = []
    for i, t in enumerate(arr):
        name = "heavy" if i % heavy_every == heavy_every - 1 else ("big" if rng.random() < 0.3 else "light")
        out.append(serving.Request(float(t), name, i))
    return out


def test_batched_server_completes_everything_within_budget():
    log = []
    tpls = make_templates(log)
    ctx = FakeCtx(0.002, tpls)
    reqs = requests(400, 4000.0, 1)
    out = serving.serve_batched(ctx, tpls, reqs, mem_budget=1000)
    assert out["completed"] == len(reqs)
    assert all(r.done >= r.arrival for r in reqs)
    # Admission: in-flight batches never held more than the budget, unless a
    # single request alone exceeds it.
    assert ctx.max_used <= 1000
    # Heavy requests never enter a batch and run on the lane's thread.
    assert all("heavy" not in names for names in ctx.submitted)
    main = threading.get_ident()
    heavy_runs = [e for e in log if e[1] == "heavy"]
    assert len(heavy_runs) == sum(r.template == "heavy" for r in reqs)
    assert all(tid != main for _, _, tid in heavy_runs)
    assert out["batches"] == len(ctx.submitted)


def test_light_requests_do_not_wait_for_the_heavy_lane():
    log = []
    tpls = make_templates(log, heavy_delay=0.2)
    ctx = FakeCtx(0.001, tpls)
    reqs = [serving.Request(0.0, "heavy", None)] + [serving.Request(0.01 + 0.001 * i, "light", i) for i in range(50)]
    serving.serve_batched(ctx, tpls, reqs, mem_budget=10**12)
    heavy = reqs[0]
    lights = reqs[1:]
    assert heavy.done >= 0.2
    assert max(r.done for r in lights) < heavy.done   # the batches went on meanwhile


def test_plain_server_runs_in_arrival_order():
    log = []
    tpls = make_templates(log, heavy_delay=0.0)
    reqs = requests(60, 20000.0, 2, heavy_every=20)
    out = serving.serve_plain(None, tpls, reqs)
    assert out["completed"] == 60
    assert [e[1] for e in log] == [r.template for r in reqs]
    assert all(reqs[i].done <= reqs[i + 1].done for i in range(len(reqs) - 1))


def test_heavy_lane_error_reaches_the_caller():
    log = []
    tpls = make_templates(log, heavy_fail=True)
    ctx = FakeCtx(0.001, tpls)
    reqs = [serving.Request(0.0, "light", 0), serving.Request(0.0, "heavy", None),
            serving.Request(0.001, "light", 1)]
    with pytest.raises(RuntimeError, match="heavy query failed"):
        serving.serve_batched(ctx, tpls, reqs, mem_budget=10**12)


def test_backlog_binds_oldest_first_and_builds_only_what_batches_need():
    """All requests arrive at once (a backlog) with two idle prepared queries:
    the queued requests are bound oldest first, each batch is submitted with
    its members in arrival order bound to their own literals, and no more
    prepared queries are built than two batches in flight and queued hold."""
    log, made = [], []

    def make():
        pq = FakePQ("light", log)
        made.append(pq)
        return pq

    tpl = serving.Template("light", make, 100)
    tpls = {"light": tpl}
    serving.reserve(tpls, 2)
    made.clear()
    ctx = FakeCtx(0.002, tpls)
    reqs = [serving.Request(0.0, "light", i) for i in range(40)]
    bound = []
    orig_submit = ctx.submit

    def submit(pqs, decode=True):
        bound.append([p.where for p in pqs])
        return orig_submit(pqs, decode)

    ctx.submit = submit
    out = serving.serve_batched(ctx, tpls, reqs, mem_budget=10**9, max_batch=8, max_inflight=1)
    assert out["completed"] == 40
    assert [w for b in bound for w in b] == list(range(40))
    assert len(made) <= 8
