"""Serving loop over resident tables: continuous batching with memory-budget
admission, against plain one-query-at-a-time execution.

Requests arrive open-loop (Poisson); each names a query template and its
literals. The batched server keeps a queue; whenever fewer than
``max_inflight`` batches are running it admits queued requests in arrival
order while their estimated device memory (group hash tables, join payloads,
result blocks) fits the budget, submits them as one ``tgp_batch_submit``, and
completes batches with ``tgp_batch_poll``. A request's latency is its
completion time minus its arrival time. The plain server runs each request
alone with ``tgp_execute`` in arrival order.
"""
from __future__ import annotations

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
    flight), each rebound to the request's predicate."""
    name: str
    make: Callable[[], PreparedQuery]
    mem_bytes: int                 # device memory a running query of this shape holds
    pool: list = field(default_factory=list)

    def take(self) -> PreparedQuery:
        return self.pool.pop() if self.pool else self.make()

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


def serve_batched(ctx: Context, templates: dict[str, Template], reqs: list[Request], mem_budget: int,
                  max_batch: int = 256, max_inflight: int = 2) -> dict:
    queue: deque[Request] = deque()
    inflight: deque = deque()      # (handle, [(req, template, pq)])
    nxt, t0 = 0, time.perf_counter()
    batches = 0
    while nxt < len(reqs) or queue or inflight:
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            queue.append(reqs[nxt])
            nxt += 1
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
                if members and used + tpl.mem_bytes > mem_budget:
                    break                    # admission: wait for memory to be released
                r = queue.popleft()
                used += tpl.mem_bytes
                members.append((r, tpl, tpl.take().rebind(r.where)))
            if members:
                inflight.append((ctx.submit([m[2] for m in members], decode=False), members))
                batches += 1
                continue
        if not queue and inflight:
            continue                         # poll again
        if not queue and nxt < len(reqs):
            wait = reqs[nxt].arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(min(wait, 0.0005))
    out = summarize(reqs, time.perf_counter() - t0)
    out["batches"] = batches
    return out


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
