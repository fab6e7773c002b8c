"""Serving loop over resident tables: continuous batching with memory-budget
admission, against plain one-query-at-a-time execution.

Requests arrive open-loop (Poisson); each names a query template and its
literals. The batched server keeps a queue; whenever fewer than
``max_inflight`` batches are running it admits queued requests in arrival
order while their estimated device memory (group hash tables, join payloads,
result blocks) fits the budget, submits them as one ``tgp_batch_submit``, and
completes batches with ``tgp_batch_poll``. Requests of a heavy template (a
high-cardinality GROUP BY, whose result is gathered, sorted and copied back
inside the call) go to a heavy lane instead: a worker thread running them one
by one on their own context, i.e. their own CUDA stream, so that the batching
loop keeps admitting and completing the light requests meanwhile. A request's
latency is its completion time minus its arrival time. The plain server runs
each request alone with ``tgp_execute`` in arrival order.
"""
from __future__ import annotations

import queue as _queue
import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from .engine import Context, PreparedQuery


@dataclass
class Request:
    arrival: float                 # seconds from the start of the run
    template: str
    where: object                  # Pred for rebind
    done: float = -1.0


@dataclass
class Template:
    """A query shape served from a pool of prepared queries (one per request in
    flight), each rebound to the request's predicate. ``mem_bytes`` is the
    device memory a running query of this shape holds: by default the
    planner's own estimate for it (``PreparedQuery.footprint``:
    tgp_query_footprint), taken from the first prepared query."""
    name: str
    make: Callable[[], PreparedQuery]
    mem_bytes: int | None = None
    pool: list = field(default_factory=list)
    heavy: bool = False            # served by the heavy lane (its prepared queries live on their own context)

    def take(self) -> PreparedQuery:
        pq = self.pool.pop() if self.pool else self.make()
        if self.mem_bytes is None:
            self.mem_bytes = int(pq.footprint())
        return pq

    def give(self, pq: PreparedQuery) -> None:
        self.pool.append(pq)


def prewarm(templates: dict[str, Template], requests: list[Request], per_template: int = 3) -> None:
    """Creates and runs ``per_template`` prepared queries of every template
    (one request's predicate each), so that the timed run neither builds
    prepared queries nor grows their output buffers (a high-cardinality
    GROUP BY resizes them to its group count on first use)."""
    for name, tpl in templates.items():
        sample = next((r for r in requests if r.template == name), None)
        where = sample.where if sample is not None else None
        pqs = [tpl.take() for _ in range(per_template)]
        for pq in pqs:
            pq.rebind(where).run(decode=False)
        for pq in pqs:
            tpl.give(pq)


def poisson_arrivals(rate: float, n: int, rng: np.random.Generator) -> np.ndarray:
    return np.cumsum(rng.exponential(1.0 / rate, n))


def summarize(reqs: list[Request], wall: float) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs if r.done >= 0])
    if lat.size == 0:
        return {"completed": 0}
    return {"completed": int(lat.size), "qps": lat.size / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3)}


class HeavyLane:
    """A worker thread that runs heavy requests one at a time, in arrival
    order, and stamps their completion times."""

    def __init__(self, t0: float):
        self.t0 = t0
        self.jobs: _queue.Queue = _queue.Queue()
        self.pending = 0
        self.error: BaseException | None = None
        self._lock = threading.Lock()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    def submit(self, r: Request, tpl: Template) -> None:
        with self._lock:
            self.pending += 1
        self.jobs.put((r, tpl))

    def busy(self) -> bool:
        with self._lock:
            return self.pending > 0

    def _run(self) -> None:
        while True:
            job = self.jobs.get()
            if job is None:
                return
            r, tpl = job
            try:
                pq = tpl.take().rebind(r.where)
                pq.run(decode=False)
                r.done = time.perf_counter() - self.t0
                tpl.give(pq)
            except BaseException as e:  # surfaced by the serving loop
                self.error = e
            with self._lock:
                self.pending -= 1

    def close(self) -> None:
        self.jobs.put(None)
        self._thread.join()


def serve_batched(ctx: Context, templates: dict[str, Template], reqs: list[Request], mem_budget: int,
                  max_batch: int = 256, max_inflight: int = 2) -> dict:
    queue: deque[Request] = deque()
    inflight: deque = deque()      # (handle, [(req, template, pq)])
    t0 = time.perf_counter()
    lane = HeavyLane(t0) if any(t.heavy for t in templates.values()) else None
    try:
        batches = _serve_loop(ctx, templates, reqs, mem_budget, max_batch, max_inflight, queue, inflight, lane, t0)
    finally:
        # On an error, batches still running are completed before returning.
        for h, _ in inflight:
            h.wait()
        if lane is not None:
            lane.close()
    if lane is not None and lane.error is not None:
        raise lane.error
    out = summarize(reqs, time.perf_counter() - t0)
    out["batches"] = batches
    return out


def _serve_loop(ctx, templates, reqs, mem_budget, max_batch, max_inflight, queue, inflight, lane, t0) -> int:
    """The batching loop of serve_batched; returns the number of batches."""
    nxt, batches = 0, 0
    while nxt < len(reqs) or queue or inflight or (lane is not None and lane.busy()):
        if lane is not None and lane.error is not None:
            break
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            r = reqs[nxt]
            nxt += 1
            if lane is not None and templates[r.template].heavy:
                lane.submit(r, templates[r.template])
            else:
                queue.append(r)
        # Complete finished batches (oldest first; they finish in order).
        while inflight and inflight[0][0].poll():
            h, members = inflight.popleft()
            t = time.perf_counter() - t0
            for r, tpl, pq in members:
                r.done = t
                tpl.give(pq)
        if queue and len(inflight) < max_inflight:
            members, used = [], sum(m[1].mem_bytes for _, ms in inflight for m in ms)
            while queue and len(members) < max_batch:
                tpl = templates[queue[0].template]
                if (members or inflight) and used + tpl.mem_bytes > mem_budget:
                    break                    # admission: wait for memory to be released
                # (A request larger than the budget runs alone once nothing else does.)
                r = queue.popleft()
                used += tpl.mem_bytes
                members.append((r, tpl, tpl.take().rebind(r.where)))
            if members:
                inflight.append((ctx.submit([m[2] for m in members], decode=False), members))
                batches += 1
                continue
        if not queue and inflight:
            continue                         # poll again
        if not queue:
            wait = reqs[nxt].arrival - (time.perf_counter() - t0) if nxt < len(reqs) else 0.0005
            if wait > 0:
                time.sleep(min(wait, 0.0005))
    return batches


def serve_plain(ctx: Context, templates: dict[str, Template], reqs: list[Request]) -> dict:
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        tpl = templates[r.template]
        pq = tpl.take().rebind(r.where)
        pq.run(decode=False)
        r.done = time.perf_counter() - t0
        tpl.give(pq)
    return summarize(reqs, time.perf_counter() - t0)
