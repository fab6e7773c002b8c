"""Serving loop over resident tables: continuous batching with memory-budget
admission, against plain one-query-at-a-time execution.

Requests arrive open-loop (Poisson) from a list, or live from a queue (the
wire front-end); each names a query template and its literals. The batched
server keeps a queue of requests, each already rebound to a prepared query of
its template when it arrived; whenever fewer than ``max_inflight`` batches are
running it admits queued requests in arrival order while the device memory their plans
need (``tgp_query_footprint``: group hash tables, join payloads, result
blocks) fits the budget, submits them as one ``tgp_batch_submit``, and
completes batches with ``tgp_batch_poll``. Requests of a heavy template (a
high-cardinality GROUP BY, whose result is gathered, sorted and copied back
inside the call) go to a heavy lane instead: a worker thread running them one
by one on their own context, i.e. their own CUDA stream, so that the batching
loop keeps admitting and completing the light requests meanwhile. A request's
latency is its completion time minus its arrival time. The plain server runs
each request alone with ``tgp_execute`` in arrival order.

A request with ``keep`` set gets its decoded result (``QueryOutput``) in
``result`` (or the exception its query raised); one with an ``event`` has it
set when done — that is how the wire front-end's connection threads wait.
"""
from __future__ import annotations

import gc
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
    keep: bool = False             # decode the result and keep it in `result`
    result: object = None          # QueryOutput, or the exception the query raised
    event: threading.Event | None = None


@dataclass
class Template:
    """A query shape served from a pool of prepared queries (one per request in
    flight), each rebound to the request's predicate. ``mem_bytes`` is the
    device memory a running query of this shape holds: by default the
    planner's own estimate for it (``PreparedQuery.footprint``:
    tgp_query_footprint), taken from the first prepared query. ``solo``, when
    set, runs a request outside the batches (ORDER BY ... LIMIT statements):
    solo(request) -> QueryOutput."""
    name: str
    make: Callable[[], PreparedQuery]
    mem_bytes: int | None = None
    pool: list = field(default_factory=list)
    heavy: bool = False            # served by the heavy lane (its prepared queries live on their own context)
    solo: Callable | None = None

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


def reserve(templates: dict[str, Template], per_template: int) -> None:
    """Grows every light template's pool of prepared queries to
    ``per_template`` (built, not run), so that a backlog of queued requests
    does not build prepared queries on the serving loop's thread."""
    for tpl in templates.values():
        if tpl.heavy or tpl.solo is not None:
            continue
        while len(tpl.pool) < per_template:
            tpl.pool.append(tpl.make())


def poisson_arrivals(rate: float, n: int, rng: np.random.Generator) -> np.ndarray:
    return np.cumsum(rng.exponential(1.0 / rate, n))


def summarize(reqs: list[Request], wall: float) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs if r.done >= 0])
    if lat.size == 0:
        return {"completed": 0}
    out = {"completed": int(lat.size), "qps": lat.size / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
           "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3)}
    per = {}
    for name in sorted({r.template for r in reqs}):
        t = np.array([r.done - r.arrival for r in reqs if r.done >= 0 and r.template == name])
        if t.size:
            per[name] = {"n": int(t.size), "p50_ms": float(np.percentile(t, 50) * 1e3),
                         "p99_ms": float(np.percentile(t, 99) * 1e3)}
    out["by_template"] = per
    return out


def freeze_heap() -> None:
    """Moves every object alive now into the collector's permanent
    generation (gc.freeze), so that the collections a serving loop triggers
    walk only the objects it creates, not the tables, pools and modules built
    before it (a full collection of those is a pause of milliseconds). Both
    servers call it when they start."""
    gc.freeze()


def _finish(r: Request, t: float, out=None, error: BaseException | None = None) -> None:
    if r.keep:
        r.result = error if error is not None else out
    r.done = t
    if r.event is not None:
        r.event.set()


# ---------------------------------------------------------------------------
# Request sources
# ---------------------------------------------------------------------------
class ListSource:
    """Requests with known arrival times (seconds from the run's start)."""

    def __init__(self, reqs: list[Request]):
        self.reqs, self.nxt = reqs, 0

    def arrived(self, now: float) -> list[Request]:
        out = []
        while self.nxt < len(self.reqs) and self.reqs[self.nxt].arrival <= now:
            out.append(self.reqs[self.nxt])
            self.nxt += 1
        return out

    def exhausted(self) -> bool:
        return self.nxt >= len(self.reqs)

    def wait(self, now: float) -> None:
        if self.nxt < len(self.reqs):
            time.sleep(min(max(self.reqs[self.nxt].arrival - now, 0.0), 0.0005))


class QueueSource:
    """Requests offered live by other threads; exhausted once closed and
    drained."""

    def __init__(self):
        self._lock = threading.Lock()
        self._items: deque[Request] = deque()
        self._ready = threading.Event()
        self.closed = False

    def offer(self, r: Request) -> None:
        with self._lock:
            self._items.append(r)
        self._ready.set()

    def close(self) -> None:
        self.closed = True
        self._ready.set()

    def arrived(self, now: float) -> list[Request]:
        with self._lock:
            out = list(self._items)
            self._items.clear()
            self._ready.clear()
        return out

    def exhausted(self) -> bool:
        with self._lock:
            return self.closed and not self._items

    def wait(self, now: float) -> None:
        self._ready.wait(timeout=0.0005)


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
                if tpl.solo is not None:
                    out = tpl.solo(r)
                else:
                    pq = tpl.take().rebind(r.where)
                    out = pq.run(decode=r.keep)
                    tpl.give(pq)
                _finish(r, time.perf_counter() - self.t0, out)
            except BaseException as e:  # surfaced by the serving loop (or to the request's waiter)
                if r.keep:
                    _finish(r, time.perf_counter() - self.t0, error=e)
                else:
                    self.error = e
            with self._lock:
                self.pending -= 1

    def close(self) -> None:
        self.jobs.put(None)
        self._thread.join()


# ---------------------------------------------------------------------------
# The batching loop
# ---------------------------------------------------------------------------
def serve_batched(ctx: Context, templates: dict[str, Template], reqs, mem_budget: int,
                  max_batch: int = 256, max_inflight: int = 2, t0: float | None = None,
                  heavy_lane: bool | None = None) -> dict:
    """Serves `reqs` (a list of Requests with arrival times, or a QueueSource
    fed live) through continuous batching until every request completed.
    `heavy_lane` (default: whether any template is heavy) starts the heavy
    lane; a live source whose templates appear later passes it explicitly."""
    source = reqs if isinstance(reqs, QueueSource) else ListSource(reqs)
    freeze_heap()
    queue: deque = deque()         # [req, template, prepared query rebound to it, or None]
    inflight: deque = deque()      # (handle, [(req, template, pq)])
    t0 = time.perf_counter() if t0 is None else t0
    if heavy_lane is None:
        heavy_lane = any(t.heavy for t in templates.values())
    lane = HeavyLane(t0) if heavy_lane else None
    seen: list[Request] = []
    try:
        batches = _serve_loop(ctx, templates, source, mem_budget, max_batch, max_inflight, queue, inflight, lane,
                              t0, seen)
    finally:
        # On an error, batches still running are completed before returning.
        for h, _ in inflight:
            h.wait()
        for _, tpl, pq in queue:
            if pq is not None:
                tpl.give(pq)
        if lane is not None:
            lane.close()
    if lane is not None and lane.error is not None:
        raise lane.error
    out = summarize(seen, time.perf_counter() - t0)
    out["batches"] = batches
    return out


def _complete(inflight: deque, t0: float, block: bool = False) -> None:
    """Completes finished batches, oldest first (they finish in order)."""
    while inflight and (inflight[0][0].poll() if not block else True):
        h, members = inflight.popleft()
        outs = h.wait()
        t = time.perf_counter() - t0
        for (r, tpl, pq), out in zip(members, outs if outs is not None else [None] * len(members)):
            _finish(r, t, out)
            tpl.give(pq)
        if block:
            return


def _serve_loop(ctx, templates, source, mem_budget, max_batch, max_inflight, queue, inflight, lane, t0,
                seen) -> int:
    """The batching loop of serve_batched; returns the number of batches."""
    batches = 0
    unbound: dict[str, deque] = {}   # per template: queued requests waiting unbound, oldest first
    while not source.exhausted() or queue or inflight or (lane is not None and lane.busy()):
        if lane is not None and lane.error is not None:
            break
        now = time.perf_counter() - t0
        for r in source.arrived(now):
            seen.append(r)
            tpl = templates[r.template]
            if lane is not None and tpl.heavy:
                lane.submit(r, tpl)
            elif tpl.solo is not None:
                # Outside the batches, on this thread (ORDER BY ... LIMIT).
                try:
                    out = tpl.solo(r)
                    _finish(r, time.perf_counter() - t0, out)
                except Exception as e:
                    if not r.keep:
                        raise
                    _finish(r, time.perf_counter() - t0, error=e)
            else:
                # Rebound on arrival, while earlier batches run, when an idle
                # prepared query is at hand and no earlier request of the
                # template waits unbound (so that a batch's members are ready
                # to submit when it is formed); otherwise when a completed
                # batch returns prepared queries, oldest request first, or at
                # admission. Admission so builds a new prepared query only
                # when a batch needs more than the pool holds.
                waiting = unbound.setdefault(tpl.name, deque())
                if tpl.pool and not waiting:
                    queue.append([r, tpl, tpl.pool.pop().rebind(r.where)])
                else:
                    entry = [r, tpl, None]
                    queue.append(entry)
                    waiting.append(entry)
        _complete(inflight, t0)
        # Prepared queries returned by completed batches go to the oldest
        # requests still waiting unbound, while the next batch runs.
        for waiting in unbound.values():
            while waiting and (waiting[0][2] is not None or waiting[0][1].pool):
                entry = waiting.popleft()
                if entry[2] is None:
                    entry[2] = entry[1].pool.pop().rebind(entry[0].where)
        if queue and len(inflight) < max_inflight:
            members, used = [], sum(m[1].mem_bytes or 0 for _, ms in inflight for m in ms)
            while queue and len(members) < max_batch:
                tpl = queue[0][1]
                if tpl.mem_bytes is None:
                    tpl.give(tpl.take())     # sizes the template from its first prepared query
                if (members or inflight) and used + tpl.mem_bytes > mem_budget:
                    break                    # admission: wait for memory to be released
                # (A request larger than the budget runs alone once nothing else does.)
                used += tpl.mem_bytes
                m = queue.popleft()
                if m[2] is None:
                    m[2] = tpl.take().rebind(m[0].where)
                members.append(tuple(m))
            if members:
                keep = any(m[0].keep for m in members)
                try:
                    h = ctx.submit([m[2] for m in members], decode=keep)
                except Exception as e:
                    if not keep:
                        raise
                    for r, tpl, pq in members:
                        _finish(r, time.perf_counter() - t0, error=e)
                        tpl.give(pq)
                    continue
                inflight.append((h, members))
                batches += 1
                continue
        if not queue and inflight:
            continue                         # poll again
        if not queue:
            source.wait(time.perf_counter() - t0)
    return batches


def serve_plain(ctx: Context, templates: dict[str, Template], reqs: list[Request]) -> dict:
    freeze_heap()
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        run_plain(templates[r.template], r, t0)
    return summarize(reqs, time.perf_counter() - t0)


def run_plain(tpl: Template, r: Request, t0: float) -> None:
    """One request alone: rebind a prepared query of its template, tgp_execute,
    stamp (and keep) the result."""
    try:
        if tpl.solo is not None:
            out = tpl.solo(r)
        else:
            pq = tpl.take().rebind(r.where)
            out = pq.run(decode=r.keep)
            tpl.give(pq)
        _finish(r, time.perf_counter() - t0, out)
    except Exception as e:
        if not r.keep:
            raise
        _finish(r, time.perf_counter() - t0, error=e)
