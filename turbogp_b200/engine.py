"""Host-side API over the C ABI: resident tables, predicates, aggregates, joins.

This mirrors what the reference's query interpreter hands to its vectorized
operators (src/engine/query_interpreter/expr.rs:419 ``build_mask``,
aggregate.rs:507 ``execute_grouped``, join.rs:544 ``hash_join_with_keys``):
a WHERE tree over typed columns, GROUP BY columns and aggregate expressions,
lowered here into the C ABI's postfix predicate program and affine-product
aggregate arguments. All compute runs in the CUDA library; nothing here falls
back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _capi as A

_NP_DTYPE = {np.dtype(np.uint8): A.DT_U8, np.dtype(np.int32): A.DT_I32, np.dtype(np.int64): A.DT_I64,
             np.dtype(np.uint64): A.DT_U64, np.dtype(np.float64): A.DT_F64}
_DT_NP = {v: k for k, v in _NP_DTYPE.items()}
_COLTYPE = {"int": A.CT_INT, "date": A.CT_DATE, "float": A.CT_FLOAT}


def _u64(v: int) -> int:
    return int(v) & 0xFFFFFFFFFFFFFFFF


# ---------------------------------------------------------------------------
# Expressions
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Factor:
    """``mul * column + add`` (column None = the constant ``add``)."""
    column: str | None
    mul: int = 1
    add: int = 0
    side: int = A.SIDE_PROBE


class Term:
    """A product of affine factors: the per-row argument of an aggregate."""

    def __init__(self, factors: Sequence[Factor]):
        self.factors = tuple(factors)

    def __mul__(self, other):
        o = _as_term(other)
        return Term(self.factors + o.factors)

    __rmul__ = __mul__

    def _affine(self) -> Factor:
        if len(self.factors) != 1:
            raise ValueError("only a single column can be offset: write (k - col) or (col + k)")
        return self.factors[0]

    def __add__(self, k):
        if isinstance(k, (Term, Col)):
            raise ValueError("sums of columns are not affine factors")
        f = self._affine()
        return Term([Factor(f.column, f.mul, f.add + int(k), f.side)])

    __radd__ = __add__

    def __sub__(self, k):
        if isinstance(k, (Term, Col)):
            raise ValueError("differences of columns are not affine factors")
        return self + (-int(k))

    def __rsub__(self, k):
        f = self._affine()
        return Term([Factor(f.column, -f.mul, int(k) - f.add, f.side)])

    def __neg__(self):
        f = self._affine()
        return Term([Factor(f.column, -f.mul, -f.add, f.side)])


class Col(Term):
    """A column reference usable in predicates and aggregate arguments."""

    def __init__(self, name: str, side: int = A.SIDE_PROBE):
        super().__init__([Factor(name, 1, 0, side)])
        self.name = name
        self.side = side

    def _leaf(self, cmp, lit, lit2=0):
        if self.side != A.SIDE_PROBE:
            raise ValueError("predicates apply to the scanned table only")
        return Pred([("leaf", self.name, cmp, lit, lit2)])

    def __eq__(self, v):  # type: ignore[override]
        return self._leaf(A.CMP_EQ, v)

    def __ne__(self, v):  # type: ignore[override]
        return self._leaf(A.CMP_NE, v)

    def __lt__(self, v):
        return self._leaf(A.CMP_LT, v)

    def __le__(self, v):
        return self._leaf(A.CMP_LE, v)

    def __gt__(self, v):
        return self._leaf(A.CMP_GT, v)

    def __ge__(self, v):
        return self._leaf(A.CMP_GE, v)

    def between(self, lo, hi):
        return self._leaf(A.CMP_BETWEEN, lo, hi)

    def not_between(self, lo, hi):
        return self._leaf(A.CMP_NOT_BETWEEN, lo, hi)

    __hash__ = object.__hash__


def col(name: str) -> Col:
    return Col(name, A.SIDE_PROBE)


def build_col(name: str) -> Col:
    """A column of the joined build table."""
    return Col(name, A.SIDE_BUILD)


def lit(k: int) -> Term:
    return Term([Factor(None, 0, int(k))])


def _as_term(x) -> Term:
    if isinstance(x, Term):
        return x
    return lit(int(x))


class Pred:
    """A WHERE tree in postfix form."""

    def __init__(self, ops):
        self.ops = list(ops)

    def __and__(self, o: "Pred") -> "Pred":
        return Pred(self.ops + o.ops + [("and",)])

    def __or__(self, o: "Pred") -> "Pred":
        return Pred(self.ops + o.ops + [("or",)])

    def __invert__(self) -> "Pred":
        return Pred(self.ops + [("not",)])


# ---------------------------------------------------------------------------
# Aggregates
# ---------------------------------------------------------------------------
@dataclass
class Agg:
    func: int
    term: Term | None = None


def count_star() -> Agg:
    return Agg(A.AGG_COUNT_STAR)


def count_col(c: Col) -> Agg:
    return Agg(A.AGG_COUNT_NONZERO, c)


def sum_(t) -> Agg:
    return Agg(A.AGG_SUM, _as_term(t))


def avg(t) -> Agg:
    return Agg(A.AGG_AVG, _as_term(t))


def min_(t) -> Agg:
    return Agg(A.AGG_MIN, _as_term(t))


def max_(t) -> Agg:
    return Agg(A.AGG_MAX, _as_term(t))


@dataclass
class AggResult:
    """One aggregate of one group: exact integer value, row count, f64 view."""
    value: int
    count: int
    as_f64: float


_AGGVALUE_DTYPE = np.dtype([("lo", "<u8"), ("hi", "<i8"), ("count", "<u8"), ("as_f64", "<f8")])


class QueryOutput:
    """Groups (key tuples) and their aggregates. A result read back from the
    device keeps its raw arrays and builds the Python lists on first access."""

    def __init__(self, keys, values, rows_scanned: int, rows_selected: int, flags: int, raw=None):
        self._keys, self._values = keys, values
        self.rows_scanned, self.rows_selected, self.flags = rows_scanned, rows_selected, flags
        self._raw = raw  # (keys u64 array, AggValue records, ngroups, nkeys, naggs)

    def _decode(self) -> None:
        keys, vals, ng, nk, na = self._raw
        kk = keys[:ng * nk].view(np.int64).reshape(ng, nk).tolist() if nk else [[] for _ in range(ng)]
        lo, hi = vals["lo"].tolist(), vals["hi"].tolist()
        cnt, f = vals["count"].tolist(), vals["as_f64"].tolist()
        self._keys = [tuple(k) for k in kk]
        self._values = [[AggResult((hi[i] << 64) | lo[i], cnt[i], f[i]) for i in range(g * na, g * na + na)]
                        for g in range(ng)]
        self._raw = None

    @property
    def keys(self) -> list[tuple[int, ...]]:
        if self._keys is None:
            self._decode()
        return self._keys

    @property
    def values(self) -> list[list[AggResult]]:
        if self._values is None:
            self._decode()
        return self._values

    @property
    def ngroups(self) -> int:
        if self._raw is not None:
            return self._raw[2]
        return len(self.values)

    def arrays(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """(keys int64 [g, k], value low limbs uint64 [g, a], value high limbs
        int64 [g, a], counts uint64 [g, a]) without building Python lists."""
        if self._raw is not None:
            keys, vals, ng, nk, na = self._raw
            k = keys[:ng * nk].view(np.int64).reshape(ng, nk)
            v = vals[:ng * na]
            return (k, v["lo"].reshape(ng, na).copy(), v["hi"].reshape(ng, na).copy(),
                    v["count"].reshape(ng, na).copy())
        ng = len(self.keys)
        nk = len(self.keys[0]) if ng else 0
        na = len(self.values[0]) if ng else 0
        k = np.array(self.keys, dtype=np.int64).reshape(ng, nk)
        lo = np.array([[x.value & 0xFFFFFFFFFFFFFFFF for x in r] for r in self.values], dtype=np.uint64).reshape(ng, na)
        hi = np.array([[x.value >> 64 for x in r] for r in self.values], dtype=np.int64).reshape(ng, na)
        cnt = np.array([[x.count for x in r] for r in self.values], dtype=np.uint64).reshape(ng, na)
        return k, lo, hi, cnt


@dataclass
class FilterOutput:
    count: int
    bitmap: np.ndarray | None = None
    rowids: np.ndarray | None = None


# ---------------------------------------------------------------------------
# Context / tables
# ---------------------------------------------------------------------------
class Context:
    """One CUDA device's execution context (tgp_init / tgp_shutdown)."""

    def __init__(self, device: int = 0):
        self.lib = A.load()
        h = C.c_void_p()
        st = self.lib.tgp_init(C.byref(h), device)
        if st != A.OK:
            raise A.TgpError(st, f"tgp_init(device={device}) failed")
        self.h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.tgp_shutdown(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int, what: str) -> None:
        if st != A.OK:
            msg = self.lib.tgp_last_error(self.h)
            raise A.TgpError(st, f"{what}: {msg.decode() if msg else ''}")

    @property
    def stream(self) -> int:
        return int(self.lib.tgp_ctx_stream(self.h) or 0)

    @property
    def sm_count(self) -> int:
        return int(self.lib.tgp_ctx_sm_count(self.h))

    def sync(self) -> None:
        self._check(self.lib.tgp_sync(self.h), "tgp_sync")

    def profile(self, on: bool = True, gated: bool = False) -> None:
        """Record CUDA events around every scan-kernel launch; with ``gated``
        each timed launch waits behind a short device delay, so the events
        bracket the kernel alone (not the host's submission of it)."""
        self._check(self.lib.tgp_profile_enable(self.h, (2 if gated else 1) if on else 0), "tgp_profile_enable")

    def profile_read(self) -> tuple[int, float]:
        """(launches, summed device ms) since the last read."""
        n, ms = C.c_uint64(), C.c_double()
        self._check(self.lib.tgp_profile_read(self.h, C.byref(n), C.byref(ms)), "tgp_profile_read")
        return int(n.value), float(ms.value)

    def register(self, columns: dict, coltypes: dict | None = None) -> "Table":
        """Copies host numpy columns into HBM. ``coltypes`` maps a name to
        'int' | 'date' | 'float' (default: 'float' for f64, else 'int')."""
        return self._register(columns, coltypes, device=False)

    def register_cells(self, cells: dict, coltypes: dict | None = None, sidecars: dict | None = None) -> "Table":
        """Registers a table in the reference's layout: one u64 cell per value
        per column (``Table::columns``), optional i32 sidecars
        (``Table::i32_columns``). The library stores each column at the
        narrowest width holding all of its values (tgp_table_register_cells).
        ``coltypes`` maps a name to 'int' | 'date' | 'float' (default 'int')."""
        coltypes, sidecars = coltypes or {}, sidecars or {}
        names = list(cells)
        descs = (A.CellColumn * max(1, len(names)))()
        keep, rows = [], None
        for i, name in enumerate(names):
            a = np.ascontiguousarray(cells[name])
            if a.dtype.itemsize != 8:
                raise TypeError(f"column {name}: cells are 8-byte words")
            keep.append(a)
            n = a.shape[0]
            descs[i].cells = a.ctypes.data
            sc = sidecars.get(name)
            if sc is not None:
                sc = np.ascontiguousarray(sc, dtype=np.int32)
                if sc.shape[0] != n:
                    raise ValueError(f"column {name}: sidecar length differs")
                keep.append(sc)
                descs[i].i32_sidecar = sc.ctypes.data
            descs[i].coltype = _COLTYPE[coltypes.get(name, "int")]
            if rows is None:
                rows = n
            elif rows != n:
                raise ValueError("columns differ in length")
        rows = rows or 0
        tid = C.c_uint64()
        self._check(self.lib.tgp_table_register_cells(self.h, descs, len(names), rows, C.byref(tid)),
                    "tgp_table_register_cells")
        dtypes = []
        for i, name in enumerate(names):
            dt = C.c_uint32()
            self._check(self.lib.tgp_table_column_dtype(self.h, tid.value, i, C.byref(dt)), "tgp_table_column_dtype")
            dtypes.append((int(dt.value), descs[i].coltype))
        return Table(self, int(tid.value), names, rows, dtypes)

    def submit(self, queries: Sequence["PreparedQuery"], decode: bool = True) -> "BatchHandle":
        """Runs prepared queries as one batch (tgp_batch_submit); a query may be
        in one unfinished batch at a time."""
        return BatchHandle(self, queries, decode)

    def register_device(self, columns: dict, coltypes: dict | None = None) -> "Table":
        """Registers device tensors (torch CUDA tensors) without copying."""
        return self._register(columns, coltypes, device=True)

    def _register(self, columns: dict, coltypes: dict | None, device: bool) -> "Table":
        coltypes = coltypes or {}
        names = list(columns)
        descs = (A.ColumnDesc * max(1, len(names)))()
        keep = []
        rows = None
        dtypes = []
        for i, name in enumerate(names):
            arr = columns[name]
            if device:
                import torch
                t = arr
                npdt = np.dtype(str(t.dtype).replace("torch.", ""))
                ptr = t.data_ptr()
                n = t.numel()
                keep.append(t)
            else:
                a = np.ascontiguousarray(arr)
                npdt = a.dtype
                ptr = a.ctypes.data
                n = a.shape[0]
                keep.append(a)
            if npdt not in _NP_DTYPE:
                raise TypeError(f"column {name}: unsupported dtype {npdt}")
            dt = _NP_DTYPE[npdt]
            ct = _COLTYPE[coltypes.get(name, "float" if dt == A.DT_F64 else "int")]
            descs[i].dtype, descs[i].coltype, descs[i].data = dt, ct, ptr
            dtypes.append((dt, ct))
            if rows is None:
                rows = n
            elif rows != n:
                raise ValueError("columns differ in length")
        rows = rows or 0
        tid = C.c_uint64()
        fn = self.lib.tgp_table_register_device if device else self.lib.tgp_table_register
        self._check(fn(self.h, descs, len(names), rows, C.byref(tid)), "tgp_table_register")
        return Table(self, int(tid.value), names, rows, dtypes, keep if device else None)

    def fail_next_scan(self, tile: int = 0, wait_ns: int = 2_000_000) -> None:
        """Test hook (tgp_debug_fail_next_scan): the next scan launch skips one
        tile's stage copy and its bounded waits give up after `wait_ns`, so
        that call raises TgpError TIMEOUT."""
        self._check(self.lib.tgp_debug_fail_next_scan(self.h, tile, wait_ns), "tgp_debug_fail_next_scan")

    def register_strings(self, values) -> "StringColumn":
        """Copies a string column into HBM (tgp_strings_register): a list of
        str / bytes, or a (uint8 bytes, uint64 offsets) pair in the flat
        layout (string i = bytes[offsets[i]:offsets[i + 1]])."""
        if isinstance(values, tuple):
            data, offs = values
        else:
            bs = [v.encode("utf-8") if isinstance(v, str) else bytes(v) for v in values]
            offs = np.zeros(len(bs) + 1, dtype=np.uint64)
            if bs:
                offs[1:] = np.cumsum([len(b) for b in bs], dtype=np.uint64)
            data = np.frombuffer(b"".join(bs), dtype=np.uint8)
        data = np.ascontiguousarray(data, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        sid = C.c_uint64()
        self._check(self.lib.tgp_strings_register(self.h, data.ctypes.data if data.size else None, data.size,
                                                  offs.ctypes.data, offs.size - 1, C.byref(sid)),
                    "tgp_strings_register")
        return StringColumn(self, int(sid.value), int(offs.size - 1))

    def join_smaller(self, a: "Table", key_a: str, where_a: "Pred | None", b: "Table", key_b: str,
                     where_b: "Pred | None") -> "JoinPlan":
        """Inner join a.key_a = b.key_b with each side's own filter, built on
        the side with fewer filtered rows (tgp_join_build_smaller, the
        reference's build-side rule)."""
        nodes_a, n_a = a.lower_pred(where_a)
        nodes_b, n_b = b.lower_pred(where_b)
        jid, on_a, ra, rb = C.c_uint64(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        self._check(self.lib.tgp_join_build_smaller(self.h, a.id, a.index(key_a), nodes_a, n_a, b.id, b.index(key_b),
                                                    nodes_b, n_b,
                                                    C.byref(jid), C.byref(on_a), C.byref(ra), C.byref(rb)),
                    "tgp_join_build_smaller")
        build, probe = (a, b) if on_a.value else (b, a)
        return JoinPlan(JoinTable(self, int(jid.value), build), probe, key_b if on_a.value else key_a,
                        where_b if on_a.value else where_a, bool(on_a.value), int(ra.value), int(rb.value))

    # -- scan variants and the autotuner --------------------------------------
    def set_default_variant(self, **knobs) -> None:
        """Sets knobs of the variant used by queries without a tuned entry
        (fields of tgp_variant: threads, max_stages, placement, presum, dense,
        shapes, payload, ctas_per_sm, l2_ahead); others keep their values."""
        v = A.Variant()
        self._check(self.lib.tgp_get_default_variant(self.h, C.byref(v)), "tgp_get_default_variant")
        for k, val in knobs.items():
            setattr(v, k, int(val))
        self._check(self.lib.tgp_set_default_variant(self.h, C.byref(v)), "tgp_set_default_variant")

    def batch_config(self, morsel_tiles: int = 16, shared_scans: bool = True, share_extra_max: int = 32768) -> None:
        self._check(self.lib.tgp_batch_config(self.h, morsel_tiles, 1 if shared_scans else 0, share_extra_max),
                    "tgp_batch_config")

    def autotune(self, pq: "PreparedQuery", reps: int = 5) -> dict:
        """Measures the scan variants of a prepared query's class
        (tgp_autotune), installs the fastest one that returns the planner's
        result bit for bit, and reports every candidate."""
        cap = 64
        entries = (A.TuneEntry * cap)()
        n, best, key = C.c_uint32(), C.c_uint32(), C.c_uint64()
        self._check(self.lib.tgp_autotune(self.h, C.byref(pq.q), reps, entries, cap, C.byref(n), C.byref(best),
                                          C.byref(key)), "tgp_autotune")
        cands = [{"variant": variant_dict(entries[i].variant), "ms": entries[i].ms, "status": entries[i].status,
                  "same_result": bool(entries[i].same_result), "threads": entries[i].threads_used,
                  "stages": entries[i].stages_used, "mode": MODE_NAMES.get(entries[i].mode_used, "?")}
                 for i in range(min(n.value, cap))]
        return {"class": int(key.value), "candidates": cands, "best": int(best.value),
                "rule_ms": cands[0]["ms"] if cands else None,
                "best_ms": cands[best.value]["ms"] if best.value < len(cands) else None}

    def tuned_variants(self) -> dict[int, dict]:
        """The tuned entries: {class key: variant fields}."""
        n = C.c_uint32()
        self._check(self.lib.tgp_tune_count(self.h, C.byref(n)), "tgp_tune_count")
        out = {}
        for i in range(n.value):
            k, v = C.c_uint64(), A.Variant()
            self._check(self.lib.tgp_tune_at(self.h, i, C.byref(k), C.byref(v)), "tgp_tune_at")
            out[int(k.value)] = variant_dict(v)
        return out

    def save_tuning(self, path) -> None:
        """Writes the tuned entries as JSON (the autotuner's cache)."""
        save_tuning_file(path, self.tuned_variants())

    def load_tuning(self, path) -> int:
        """Installs the entries of a JSON cache written by save_tuning;
        returns how many."""
        entries = load_tuning_file(path)
        for key, fields in entries.items():
            v = A.Variant()
            for f, val in fields.items():
                setattr(v, f, int(val))
            self._check(self.lib.tgp_tune_set(self.h, key, C.byref(v)), "tgp_tune_set")
        return len(entries)

    # -- kernel-table boundary ------------------------------------------------
    def kernel_execute(self, op: int, input_ptr: int, output_ptr: int | None, params: A.KernelParams):
        r = A.KernelResultC()
        self._check(self.lib.tgp_kernel_execute(self.h, op, input_ptr, output_ptr, C.byref(params), C.byref(r)),
                    "tgp_kernel_execute")
        return r

    def hash_table_free(self, handle: int) -> None:
        self._check(self.lib.tgp_hash_table_free(self.h, C.c_void_p(handle)), "tgp_hash_table_free")


MODE_NAMES = {2: "private", 3: "shared", 4: "global", 5: "hash", 8: "shared32"}
VARIANT_FIELDS = ("threads", "max_stages", "placement", "presum", "dense", "shapes", "payload", "ctas_per_sm",
                  "l2_ahead")


def variant_dict(v) -> dict:
    return {f: int(getattr(v, f)) for f in VARIANT_FIELDS}


def save_tuning_file(path, entries: dict) -> None:
    """The autotuner's cache: {"version": 1, "entries": [{"class": key,
    "variant": {...}}, ...]} in ascending class order."""
    import json
    doc = {"version": 1, "entries": [{"class": int(k), "variant": {f: int(v[f]) for f in VARIANT_FIELDS}}
                                     for k, v in sorted(entries.items())]}
    with open(path, "w") as fh:
        json.dump(doc, fh, indent=1)


def load_tuning_file(path) -> dict:
    import json
    with open(path) as fh:
        doc = json.load(fh)
    if doc.get("version") != 1:
        raise ValueError("unknown tuning cache version")
    out = {}
    for e in doc["entries"]:
        v = e["variant"]
        unknown = set(v) - set(VARIANT_FIELDS)
        if unknown:
            raise ValueError(f"unknown variant fields {sorted(unknown)}")
        out[int(e["class"])] = {f: int(v.get(f, 0)) for f in VARIANT_FIELDS}
    return out


def string_cell(v: str | bytes) -> int:
    """The cell of a string value as the reference stores it: xxh3_64 of its
    UTF-8 bytes (src/datasource/parquet.rs:389-406; equality predicates hash
    their literal the same way, expr.rs:1534-1547)."""
    try:
        import xxhash
    except ImportError as e:  # pragma: no cover - the package ships with the image
        raise ImportError("string values need the xxhash package (xxh3_64)") from e
    return int(xxhash.xxh3_64_intdigest(v.encode("utf-8") if isinstance(v, str) else bytes(v)))


def _lit_bits(ct: int, v) -> int:
    if isinstance(v, (str, bytes)):
        return string_cell(v)
    if ct == A.CT_FLOAT:
        return int(np.array([float(v)], dtype=np.float64).view(np.uint64)[0])
    return _u64(int(v))


class Schema:
    """Column names and (dtype, coltype) pairs; lowers expressions to C-ABI structs."""

    def __init__(self, names, dtypes):
        self.names = list(names)
        self.dtypes = list(dtypes)
        self._index = {n: i for i, n in enumerate(self.names)}

    @classmethod
    def of(cls, columns: dict, coltypes: dict | None = None) -> "Schema":
        coltypes = coltypes or {}
        dts = []
        for name, a in columns.items():
            dt = _NP_DTYPE[np.dtype(a.dtype)]
            dts.append((dt, _COLTYPE[coltypes.get(name, "float" if dt == A.DT_F64 else "int")]))
        return cls(list(columns), dts)

    def index(self, name: str) -> int:
        try:
            return self._index[name]
        except KeyError:
            raise KeyError(f"unknown column {name!r}") from None

    def lower_pred(self, pred: Pred | None):
        if pred is None or not pred.ops:
            return None, 0
        nodes = (A.PredNode * len(pred.ops))()
        for i, op in enumerate(pred.ops):
            if op[0] == "leaf":
                _, name, cmp, v, v2 = op
                if isinstance(v, (str, bytes)) and cmp not in (A.CMP_EQ, A.CMP_NE):
                    raise ValueError("string values compare by equality only (their cells are xxh3_64 hashes)")
                ci = self.index(name)
                ct = self.dtypes[ci][1]
                nodes[i].kind, nodes[i].column, nodes[i].cmp = A.PN_LEAF, ci, cmp
                nodes[i].lit = _lit_bits(ct, v)
                nodes[i].lit2 = _lit_bits(ct, v2)
            else:
                nodes[i].kind = {"and": A.PN_AND, "or": A.PN_OR, "not": A.PN_NOT}[op[0]]
        return nodes, len(pred.ops)

    def _lower_term(self, term: Term | None, agg: A.Agg, build: "Schema | None") -> None:
        factors = term.factors if term is not None else ()
        if len(factors) > A.MAX_FACTORS:
            raise ValueError("at most 4 factors per aggregate")
        agg.nfactors = len(factors)
        for j, f in enumerate(factors):
            if f.column is None:
                agg.f[j].column = -1
            elif f.side == A.SIDE_BUILD:
                if build is None:
                    raise ValueError("build-side column without a join")
                agg.f[j].column = build.index(f.column)
            else:
                agg.f[j].column = self.index(f.column)
            agg.f[j].side = f.side
            agg.f[j].mul = f.mul
            agg.f[j].add = f.add

    def lower_query(self, aggs: Sequence[Agg], group_by=(), where: Pred | None = None,
                    build: "Schema | None" = None, probe_key: str | None = None):
        """Returns (tgp_query, keepalive); q.table and q.join are left 0."""
        nodes, npred = self.lower_pred(where)
        q = A.Query()
        q.pred = nodes if nodes is not None else None
        q.npred = npred
        gk = (A.GroupKey * max(1, len(group_by)))()
        for i, g in enumerate(group_by):
            c_ = g if isinstance(g, Col) else col(g)
            if c_.side == A.SIDE_BUILD:
                if build is None:
                    raise ValueError("build-side group key without a join")
                gk[i].column = build.index(c_.name)
            else:
                gk[i].column = self.index(c_.name)
            gk[i].side = c_.side
        q.ngroup = len(group_by)
        q.group = gk
        ag = (A.Agg * max(1, len(aggs)))()
        for i, a in enumerate(aggs):
            ag[i].func = a.func
            self._lower_term(a.term, ag[i], build)
        q.nagg = len(aggs)
        q.aggs = ag
        if probe_key is not None:
            q.probe_key_column = self.index(probe_key)
        return q, (nodes, gk, ag)


def decode_groups(keys: np.ndarray, vals, ngroups: int, nkeys: int, naggs: int):
    out_keys, out_vals = [], []
    for g in range(ngroups):
        out_keys.append(tuple(int(np.int64(keys[g * nkeys + k])) for k in range(nkeys)))
        row = []
        for a in range(naggs):
            v = vals[g * naggs + a]
            row.append(AggResult(v.value, int(v.count), float(v.as_f64)))
        out_vals.append(row)
    return out_keys, out_vals


class Table(Schema):
    def __init__(self, ctx: Context, tid: int, names, rows, dtypes, keepalive=None):
        super().__init__(names, dtypes)
        self.ctx, self.id, self.rows = ctx, tid, rows
        self._keep = keepalive

    def drop(self) -> None:
        if self.id:
            self.ctx._check(self.ctx.lib.tgp_table_drop(self.ctx.h, self.id), "tgp_table_drop")
            self.id = 0

    def stats(self, name: str) -> tuple[int, int]:
        lo, hi = C.c_int64(), C.c_int64()
        self.ctx._check(self.ctx.lib.tgp_table_column_stats(self.ctx.h, self.id, self.index(name), C.byref(lo),
                                                            C.byref(hi)), "tgp_table_column_stats")
        return lo.value, hi.value

    def reload(self, columns: dict) -> None:
        descs = (A.ColumnDesc * len(self.names))()
        keep = []
        for i, name in enumerate(self.names):
            a = np.ascontiguousarray(columns[name])
            keep.append(a)
            descs[i].dtype, descs[i].coltype, descs[i].data = self.dtypes[i][0], self.dtypes[i][1], a.ctypes.data
        self.ctx._check(self.ctx.lib.tgp_table_reload(self.ctx.h, self.id, descs, len(self.names)), "tgp_table_reload")

    # -- operations -----------------------------------------------------------
    def filter(self, where: Pred | None, bitmap: bool = True, rowids: bool = True) -> FilterOutput:
        nodes, n = self.lower_pred(where)
        cnt = C.c_uint64()
        bm = np.zeros((self.rows + 7) // 8, dtype=np.uint8) if bitmap else None
        rid = np.zeros(max(1, self.rows), dtype=np.uint32) if rowids else None
        self.ctx._check(self.ctx.lib.tgp_filter(
            self.ctx.h, self.id, nodes, n,
            bm.ctypes.data if bm is not None and bm.size else None,
            rid.ctypes.data if rid is not None else None,
            self.rows if rowids else 0, C.byref(cnt)), "tgp_filter")
        c = int(cnt.value)
        return FilterOutput(c, bm, rid[:c].copy() if rid is not None else None)

    def prepare(self, aggs: Sequence[Agg], group_by: Sequence[Col | str] = (), where: Pred | None = None,
                join: "JoinTable | None" = None, probe_key: str | None = None,
                group_cap: int = 1024) -> "PreparedQuery":
        """Lowers a query once; ``run()`` executes it with no per-call lowering."""
        return PreparedQuery(self, aggs, group_by, where, join, probe_key, group_cap)

    def aggregate(self, aggs: Sequence[Agg], group_by: Sequence[Col | str] = (), where: Pred | None = None,
                  join: "JoinTable | None" = None, probe_key: str | None = None,
                  group_cap: int | None = None) -> QueryOutput:
        return self.prepare(aggs, group_by, where, join, probe_key, group_cap or 1024).run()

    def aggregate_topn(self, aggs: Sequence[Agg], group_by: Sequence[Col | str], where: Pred | None, order_by: int,
                       descending: bool, limit: int, join: "JoinTable | None" = None,
                       probe_key: str | None = None) -> QueryOutput:
        """GROUP BY ... ORDER BY aggs[order_by] [DESC] LIMIT limit
        (tgp_execute_topn): at most ``limit`` groups in the aggregate's order,
        ties in ascending key order."""
        build = join.build if join is not None else None
        q, keep = self.lower_query(aggs, group_by, where, build, probe_key)
        q.table = self.id
        if join is not None:
            q.join = join.id
        nk, na = len(group_by), len(aggs)
        keys = np.zeros(max(1, limit * max(1, nk)), dtype=np.uint64)
        vals = (A.AggValue * max(1, limit * max(1, na)))()
        res = A.QueryResult()
        self.ctx._check(self.ctx.lib.tgp_execute_topn(self.ctx.h, C.byref(q), order_by, 1 if descending else 0, limit,
                                                      keys.ctypes.data, vals, C.byref(res)), "tgp_execute_topn")
        ks, vs = decode_groups(keys, vals, int(res.ngroups), nk, na)
        return QueryOutput(ks, vs, int(res.rows_scanned), int(res.rows_selected), int(res.flags))

    def count_distinct(self, column: str, where: Pred | None = None) -> tuple[int, str]:
        """COUNT(DISTINCT column) [WHERE where] (tgp_count_distinct): (count,
        'exact' | 'hll'), exact below 100,000 selected rows as in the reference."""
        nodes, n = self.lower_pred(where)
        cnt, method = C.c_uint64(), C.c_uint32()
        self.ctx._check(self.ctx.lib.tgp_count_distinct(self.ctx.h, self.id, self.index(column), nodes, n,
                                                        C.byref(cnt), C.byref(method)), "tgp_count_distinct")
        return int(cnt.value), ("hll" if method.value else "exact")

    def join_build(self, key: str, where: Pred | None = None) -> "JoinTable":
        nodes, n = self.lower_pred(where)
        jid = C.c_uint64()
        self.ctx._check(self.ctx.lib.tgp_join_build(self.ctx.h, self.id, self.index(key), nodes, n, C.byref(jid)),
                        "tgp_join_build")
        return JoinTable(self.ctx, int(jid.value), self)


class PreparedQuery:
    """A lowered tgp_query with its output buffers (tgp_execute per ``run``)."""

    def __init__(self, table: Table, aggs, group_by, where, join, probe_key, group_cap: int):
        build = join.build if join is not None else None
        self.table = table
        self.q, self._keep = table.lower_query(aggs, group_by, where, build, probe_key)
        self.q.table = table.id
        if join is not None:
            self.q.join = join.id
        self.nk, self.na = len(group_by), len(aggs)
        # The query as written (checkers and the serving loop re-read it).
        self.spec = {"aggs": list(aggs), "group_by": tuple(group_by), "where": where, "join": join,
                     "probe_key": probe_key}
        self._alloc(group_cap)
        self.res = A.QueryResult()
        self._fn = table.ctx.lib.tgp_execute
        self.graph = 0

    def footprint(self) -> int:
        """Device bytes one run of this query holds while it runs, as its plan
        sizes them (tgp_query_footprint): result block, group hash table and
        the buffers of its result, a join payload still to be built."""
        ctx = self.table.ctx
        b = C.c_uint64()
        ctx._check(ctx.lib.tgp_query_footprint(ctx.h, C.byref(self.q), C.byref(b)), "tgp_query_footprint")
        return int(b.value)

    def rebind(self, where: Pred | None) -> "PreparedQuery":
        """Replaces the WHERE program (new literals or shape); the rest of the
        lowered query and the output buffers are kept."""
        nodes, n = self.table.lower_pred(where)
        self.q.pred = nodes if nodes is not None else None
        self.q.npred = n
        self._keep = (nodes,) + tuple(self._keep[1:])
        self.spec["where"] = where
        if self.graph:
            self.capture()
        return self

    def capture(self) -> "PreparedQuery":
        """Records the query as a CUDA graph (tgp_graph_capture); later ``run``
        calls replay it with one graph launch and no planning. Direct-indexed
        and scalar aggregates only (a hash-grouped query raises TgpError
        UNSUPPORTED)."""
        ctx = self.table.ctx
        self.drop_graph()
        gid = C.c_uint64()
        ctx._check(ctx.lib.tgp_graph_capture(ctx.h, C.byref(self.q), C.byref(gid)), "tgp_graph_capture")
        self.graph = int(gid.value)
        return self

    def drop_graph(self) -> None:
        if self.graph:
            ctx = self.table.ctx
            gid, self.graph = self.graph, 0
            ctx._check(ctx.lib.tgp_graph_drop(ctx.h, gid), "tgp_graph_drop")

    # Output buffers of at least this many bytes are page-locked, so the
    # device-to-host copy of a large grouped result runs at full link speed.
    PINNED_BYTES = 16 << 20

    def _alloc(self, cap: int) -> None:
        self.cap = cap
        nkeys, nvals = max(1, cap * max(1, self.nk)), max(1, cap * max(1, self.na))
        vbytes = nvals * C.sizeof(A.AggValue)
        if 8 * nkeys + vbytes >= self.PINNED_BYTES:
            import torch  # page-locked host memory from torch's caching host allocator
            self._pinned = (torch.empty(8 * nkeys, dtype=torch.uint8, pin_memory=True),
                            torch.empty(vbytes, dtype=torch.uint8, pin_memory=True))
            self.keys = self._pinned[0].numpy().view(np.uint64)
            self.vals = (A.AggValue * nvals).from_buffer(self._pinned[1].numpy())
        else:
            self._pinned = None
            self.keys = np.zeros(nkeys, dtype=np.uint64)
            self.vals = (A.AggValue * nvals)()
        self._vals_np = np.frombuffer(self.vals, dtype=_AGGVALUE_DTYPE)

    def run(self, decode: bool = True) -> QueryOutput:
        """Executes the query; with decode=False only the counts are returned
        (the raw results stay in ``keys`` / ``vals``)."""
        ctx = self.table.ctx
        while True:
            if self.graph:
                st = ctx.lib.tgp_graph_launch(ctx.h, self.graph, self.keys.ctypes.data, self.vals, self.cap,
                                              C.byref(self.res))
            else:
                st = self._fn(ctx.h, C.byref(self.q), self.keys.ctypes.data, self.vals, self.cap, C.byref(self.res))
            if st == A.CAPACITY and self.res.ngroups > self.cap:
                self._alloc(int(self.res.ngroups))
                continue
            ctx._check(st, "tgp_graph_launch" if self.graph else "tgp_execute")
            break
        return self._output(self.res, decode)

    def _output(self, r, decode: bool = True) -> QueryOutput:
        if not decode:
            return QueryOutput([], [], int(r.rows_scanned), int(r.rows_selected), int(r.flags))
        ng = int(r.ngroups)
        raw = (self.keys[:ng * self.nk].copy(), self._vals_np[:ng * self.na].copy(), ng, self.nk, self.na)
        return QueryOutput(None, None, int(r.rows_scanned), int(r.rows_selected), int(r.flags), raw)


class BatchHandle:
    """Queries submitted together with tgp_batch_submit (one persistent launch
    for the direct / scalar aggregates). ``poll()`` is non-blocking; ``wait()``
    returns one QueryOutput per query, in submission order."""

    def __init__(self, ctx: Context, queries: Sequence["PreparedQuery"], decode: bool = True):
        self.ctx, self.queries, self.decode = ctx, list(queries), decode
        self.items = (A.BatchItem * max(1, len(self.queries)))()
        for i, pq in enumerate(self.queries):
            it = self.items[i]
            it.query = C.pointer(pq.q)
            it.keys_out = pq.keys.ctypes.data
            it.vals_out = pq.vals
            it.group_cap = pq.cap
        bid = C.c_uint64()
        ctx._check(ctx.lib.tgp_batch_submit(ctx.h, self.items, len(self.queries), C.byref(bid)), "tgp_batch_submit")
        self.id = int(bid.value)
        self.outputs: list[QueryOutput] | None = None

    def _finish(self) -> None:
        outs = []
        for i, pq in enumerate(self.queries):
            it = self.items[i]
            if it.status == A.CAPACITY:
                outs.append(pq.run(self.decode))  # more groups than the buffer: rerun alone, resized
                continue
            if it.status != A.OK:
                self.ctx._check(it.status, f"batch query {i}")
            outs.append(pq._output(it.result, self.decode))
        self.outputs = outs

    def poll(self) -> bool:
        if self.outputs is not None:
            return True
        st = self.ctx.lib.tgp_batch_poll(self.ctx.h, self.id, 0)
        if st == A.PENDING:
            return False
        self.ctx._check(st, "tgp_batch_poll")
        self._finish()
        return True

    def wait(self) -> list[QueryOutput]:
        if self.outputs is None:
            self.ctx._check(self.ctx.lib.tgp_batch_poll(self.ctx.h, self.id, 1), "tgp_batch_poll")
            self._finish()
        return self.outputs


class JoinTable:
    def __init__(self, ctx: Context, jid: int, build: Table):
        self.ctx, self.id, self.build = ctx, jid, build

    def drop(self) -> None:
        if self.id:
            self.ctx._check(self.ctx.lib.tgp_join_drop(self.ctx.h, self.id), "tgp_join_drop")
            self.id = 0

    def probe_pairs(self, probe: Table, probe_key: str, where: Pred | None = None):
        nodes, n = probe.lower_pred(where)
        npairs = C.c_uint64()
        st = self.ctx.lib.tgp_join_probe_pairs(self.ctx.h, self.id, probe.id, probe.index(probe_key), nodes, n,
                                               None, None, 0, C.byref(npairs))
        if st not in (A.OK, A.CAPACITY):
            self.ctx._check(st, "tgp_join_probe_pairs")
        m = int(npairs.value)
        pr = np.zeros(max(1, m), dtype=np.uint32)
        br = np.zeros(max(1, m), dtype=np.uint32)
        if m:
            self.ctx._check(self.ctx.lib.tgp_join_probe_pairs(
                self.ctx.h, self.id, probe.id, probe.index(probe_key), nodes, n, pr.ctypes.data, br.ctypes.data, m,
                C.byref(npairs)), "tgp_join_probe_pairs")
        return pr[:m], br[:m]


def _flip_side(side: int) -> int:
    return A.SIDE_BUILD if side == A.SIDE_PROBE else A.SIDE_PROBE


def _flip_agg(a: Agg) -> Agg:
    if a.term is None:
        return Agg(a.func, None)
    return Agg(a.func, Term([Factor(f.column, f.mul, f.add, _flip_side(f.side) if f.column is not None else f.side)
                             for f in a.term.factors]))


def _flip_key(k) -> Col:
    c = k if isinstance(k, Col) else col(k)
    return Col(c.name, _flip_side(c.side))


@dataclass
class JoinPlan:
    """An inner join whose build side was chosen by row counts
    (Context.join_smaller). Queries are written with table a's columns as
    ``col`` and table b's as ``build_col``; when a was the smaller side (and
    so was built), the sides are swapped before execution."""
    join: JoinTable
    probe: Table
    probe_key: str
    probe_where: Pred | None
    build_is_a: bool
    rows_a: int
    rows_b: int

    def aggregate(self, aggs: Sequence[Agg], group_by: Sequence = (), group_cap: int | None = None) -> QueryOutput:
        if self.build_is_a:
            aggs = [_flip_agg(a) for a in aggs]
            group_by = [_flip_key(k) for k in group_by]
        return self.probe.aggregate(aggs, group_by, self.probe_where, join=self.join, probe_key=self.probe_key,
                                    group_cap=group_cap)

    def pairs(self) -> tuple[np.ndarray, np.ndarray]:
        """(row of a, row of b) index pairs in (probe row, build row) order."""
        pr, br = self.join.probe_pairs(self.probe, self.probe_key, self.probe_where)
        return (br, pr) if self.build_is_a else (pr, br)

    def drop(self) -> None:
        self.join.drop()


class StringColumn:
    """A string column resident in HBM (flat bytes + offsets)."""

    def __init__(self, ctx: Context, sid: int, n: int):
        self.ctx, self.id, self.n = ctx, sid, n

    def like(self, pattern: str | bytes, negated: bool = False) -> FilterOutput:
        """``col [NOT] LIKE pattern``: (count, LSB-first selection bitmap) —
        AND the bitmap into a WHERE bitmap (``Table.filter``) as the
        reference does."""
        p = pattern.encode("utf-8") if isinstance(pattern, str) else bytes(pattern)
        bm = np.zeros(max(1, (self.n + 7) // 8), dtype=np.uint8)
        cnt = C.c_uint64()
        self.ctx._check(self.ctx.lib.tgp_like(self.ctx.h, self.id, p, len(p), 1 if negated else 0, bm.ctypes.data,
                                              C.byref(cnt)), "tgp_like")
        return FilterOutput(int(cnt.value), bm[:(self.n + 7) // 8])

    def drop(self) -> None:
        if self.id:
            self.ctx._check(self.ctx.lib.tgp_strings_drop(self.ctx.h, self.id), "tgp_strings_drop")
            self.id = 0
