"""SQL statements from the wire front-end, executed by the serving loop.

``Frontend`` holds the catalog (tables registered by name, with the context
they live on), lowers each statement (``sqlfront.parse``), keeps one serving
``Template`` per statement shape — statements that differ only in probe-side
WHERE literals share prepared queries, rebound per statement — and builds join
tables per (build table, build key, build WHERE) once. Two executors run the
statements:

* ``BatchingExecutor`` — a dispatcher thread running the continuous-batching
  loop (``serving.serve_batched`` over a live ``QueueSource``); statements over
  tables registered ``heavy`` run in its heavy lane on their own context;
* ``PlainExecutor`` — one statement at a time in arrival order, each with its
  own ``tgp_execute`` (the plain per-query-launch path).

Both have ``execute(sql) -> (column names, rows of text)`` for
``pgwire.PgWireServer``; a connection thread blocks only on its own statement.
"""
from __future__ import annotations

import threading
import time
from collections import deque

from . import serving, sqlfront
from .engine import Context, Table


class Frontend:
    def __init__(self, ctx: Context, heavy_ctx: Context | None = None):
        self.ctx, self.heavy_ctx = ctx, heavy_ctx
        self.tables: dict[str, tuple[Table, bool]] = {}
        self.catalog: dict[str, sqlfront.TableInfo] = {}
        self.templates: dict[str, serving.Template] = {}
        self.specs: dict[str, sqlfront.QuerySpec] = {}
        self.joins: dict[tuple, object] = {}
        self._lock = threading.Lock()

    def register(self, name: str, columns: dict, coltypes: dict | None = None, heavy: bool = False) -> Table:
        """Registers host columns under `name` (on the heavy context when
        `heavy`: statements over it run in the heavy lane)."""
        ctx = self.heavy_ctx if heavy and self.heavy_ctx is not None else self.ctx
        t = ctx.register(columns, coltypes)
        return self.add_table(name, t, coltypes, heavy)

    def add_table(self, name: str, table: Table, coltypes: dict | None = None, heavy: bool = False) -> Table:
        self.tables[name] = (table, heavy)
        self.catalog[name] = sqlfront.TableInfo(name, list(table.names), dict(coltypes or {}))
        return table

    def close(self) -> None:
        for j in self.joins.values():
            j.drop()
        self.joins.clear()
        for tpl in self.templates.values():
            tpl.pool.clear()

    # -- statements -------------------------------------------------------------
    def request(self, sql: str, arrival: float = 0.0) -> tuple[serving.Request, sqlfront.QuerySpec]:
        """Parses a statement and returns its serving request (keep = True)
        and lowered form; creates the statement shape's template on first use."""
        spec = sqlfront.parse(sql, self.catalog)
        with self._lock:
            if spec.shape not in self.templates:
                self.templates[spec.shape] = self._template(spec)
                self.specs[spec.shape] = spec
        return serving.Request(arrival, spec.shape, spec.where, keep=True), spec

    def _join(self, spec: sqlfront.QuerySpec):
        btable, bkey, _, bwhere = spec.join
        key = (btable, bkey, repr(bwhere.ops) if bwhere is not None else None)
        if key not in self.joins:
            table, _ = self.tables[btable]
            self.joins[key] = table.join_build(bkey, bwhere)
        return self.joins[key]

    def _template(self, spec: sqlfront.QuerySpec) -> serving.Template:
        """The serving template of a statement shape. Nothing here touches the
        GPU: a context is used by one thread at a time, so the join table is
        built by `make` / `solo`, which run on the serving loop's thread (or
        the heavy lane's, for tables on the heavy context)."""
        table, heavy = self.tables[spec.table]
        probe_key = spec.join[2] if spec.join else None
        if spec.join and self.tables[spec.join[0]][1] != heavy:
            raise sqlfront.SqlError("0A000", "a join between tables on different contexts")
        join = (lambda: self._join(spec)) if spec.join else (lambda: None)
        make = lambda: table.prepare(spec.aggs, spec.group_by, spec.where, join=join(), probe_key=probe_key,
                                     group_cap=1 << 16)
        solo = None
        if spec.order is not None:
            agg, desc = spec.order
            solo = lambda r: table.aggregate_topn(spec.aggs, spec.group_by, r.where, agg, desc, spec.limit,
                                                  join=join(), probe_key=probe_key)
        return serving.Template(spec.shape, make, heavy=heavy, solo=solo)

    def rows(self, spec: sqlfront.QuerySpec, r: serving.Request) -> tuple[list[str], list[tuple]]:
        if isinstance(r.result, BaseException):
            err = r.result
            if isinstance(err, sqlfront.SqlError):
                raise err
            raise sqlfront.SqlError("XX000", f"{type(err).__name__}: {err}")
        return sqlfront.format_rows(spec, r.result)


class BatchingExecutor:
    """Statements served by the continuous-batching loop on a dispatcher
    thread (started by start(), ended by stop())."""

    def __init__(self, fe: Frontend, mem_budget: int = 8 << 30, max_batch: int = 256, max_inflight: int = 2):
        self.fe, self.mem_budget, self.max_batch, self.max_inflight = fe, mem_budget, max_batch, max_inflight
        self.source = serving.QueueSource()
        self.t0 = time.perf_counter()
        self.stats: dict | None = None
        self.error: BaseException | None = None
        self._thread = threading.Thread(target=self._run, daemon=True)

    def start(self) -> "BatchingExecutor":
        self._thread.start()
        return self

    def _run(self) -> None:
        try:
            self.stats = serving.serve_batched(self.fe.ctx, self.fe.templates, self.source, self.mem_budget,
                                               self.max_batch, self.max_inflight, t0=self.t0,
                                               heavy_lane=self.fe.heavy_ctx is not None)
        except BaseException as e:   # reported to stop()'s caller
            self.error = e

    def execute(self, sql: str):
        r, spec = self.fe.request(sql, time.perf_counter() - self.t0)
        r.event = threading.Event()
        self.source.offer(r)
        if not r.event.wait(timeout=300.0):
            raise sqlfront.SqlError("57014", "statement timed out in the serving queue")
        return self.fe.rows(spec, r)

    def stop(self) -> dict | None:
        self.source.close()
        self._thread.join()
        if self.error is not None:
            raise self.error
        return self.stats


class PlainExecutor:
    """Statements run one at a time, in arrival order, each alone on the GPU."""

    def __init__(self, fe: Frontend):
        self.fe = fe
        self.t0 = time.perf_counter()
        self._q: deque = deque()
        self._cv = threading.Condition()
        self._stop = False
        self._thread = threading.Thread(target=self._run, daemon=True)

    def start(self) -> "PlainExecutor":
        self._thread.start()
        return self

    def _run(self) -> None:
        while True:
            with self._cv:
                while not self._q and not self._stop:
                    self._cv.wait()
                if not self._q:
                    return
                r = self._q.popleft()
            serving.run_plain(self.fe.templates[r.template], r, self.t0)

    def execute(self, sql: str):
        r, spec = self.fe.request(sql, time.perf_counter() - self.t0)
        r.event = threading.Event()
        with self._cv:
            self._q.append(r)
            self._cv.notify()
        r.event.wait()
        return self.fe.rows(spec, r)

    def stop(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()
