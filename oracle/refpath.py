"""TEST / BASELINE INFRASTRUCTURE: Python driver of ``ref_path.cpp`` (the C++
restatement of the reference's CPU execution of the benchmark queries)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import load


class RefLeaf(C.Structure):
    _fields_ = [("col", C.c_uint32), ("op", C.c_uint32), ("sgn", C.c_uint32), ("_pad", C.c_uint32),
                ("lit", C.c_uint64), ("lit2", C.c_uint64)]


_OPS = {0: 0, 1: 1, 2: 2, 3: 3, 4: 4, 5: 5, 6: 6}  # tgp_cmp -> ref op (BETWEEN = 6)
COLTYPES = {"ship_day": "date", "discount_pct": "int", "quantity": "int", "price_cents": "int"}


def to_cells(a: np.ndarray) -> np.ndarray:
    """The reference's storage: one u64 cell per value (sign-extended)."""
    return a.astype(np.int64).view(np.uint64) if a.dtype != np.uint64 else a


def selective_scan_sum(cols: dict, tpl, threads: int | None = None) -> dict:
    """Runs the conjunction + SUM(a*b) + COUNT template the reference's way.

    ``cols`` holds native-width numpy columns; they are widened to u64 cells
    outside the timed region (that is the reference's table layout)."""
    lib = load()
    fn = lib.ref_scan_sum_mul
    fn.restype = C.c_double
    fn.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.POINTER(RefLeaf), C.c_uint32, C.c_uint32, C.c_uint32,
                   C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    names = list(cols)
    cells = [np.ascontiguousarray(to_cells(cols[n])) for n in names]
    ptrs = (C.c_void_p * len(cells))(*[c.ctypes.data for c in cells])
    leaves = []
    for op in tpl.where.ops:
        if op[0] == "and":
            continue
        if op[0] != "leaf":
            raise ValueError("the scan baseline takes a conjunction of leaves")
        _, name, cmp, v, v2 = op
        L = RefLeaf()
        L.col, L.op = names.index(name), _OPS[cmp]
        L.sgn = 1 if COLTYPES.get(name, "int") == "int" else 0
        L.lit, L.lit2 = int(v) & 0xFFFFFFFFFFFFFFFF, int(v2) & 0xFFFFFFFFFFFFFFFF
        leaves.append(L)
    arr = (RefLeaf * len(leaves))(*leaves)
    (f_a, f_b) = tpl.aggs[0].term.factors
    s, c = C.c_double(), C.c_uint64()
    sec = fn(ptrs, cells[0].shape[0], arr, len(leaves), names.index(f_a.column), names.index(f_b.column),
             C.byref(s), C.byref(c))
    return {"seconds": sec, "sum": s.value, "count": int(c.value), "threads": 1}


def _leaves(names: list, where, coltypes: dict):
    leaves = []
    for op in (where.ops if where is not None else []):
        if op[0] == "and":
            continue
        if op[0] != "leaf":
            raise ValueError("the baseline takes a conjunction of leaves")
        _, name, cmp, v, v2 = op
        L = RefLeaf()
        L.col, L.op = names.index(name), _OPS[cmp]
        L.sgn = 1 if coltypes.get(name, "int") == "int" else 0
        L.lit, L.lit2 = int(v) & 0xFFFFFFFFFFFFFFFF, int(v2) & 0xFFFFFFFFFFFFFFFF
        leaves.append(L)
    return (RefLeaf * max(1, len(leaves)))(*leaves), len(leaves)


def grouped_q1(cols: dict, tpl, coltypes: dict, threads: int | None = None) -> dict:
    """The filtered grouped aggregate (GROUP BY flag_a, flag_b: count, sum(quantity),
    sum(price), sum(price*(100-disc)), sum(price*(100-disc)*(100+tax)),
    avg(quantity)) the reference's way (``ref_grouped_q1``). Returns the wall
    seconds and the groups sorted by key: (keys, count, sum_q, sum_p,
    disc_price f64, charge f64, avg_q f64)."""
    import os
    lib = load()
    fn = lib.ref_grouped_q1
    fn.restype = C.c_double
    fn.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.POINTER(RefLeaf), C.c_uint32] + [C.c_uint32] * 6 + \
        [C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]
    names = list(cols)
    cells = [np.ascontiguousarray(to_cells(cols[n])) for n in names]
    ptrs = (C.c_void_p * len(cells))(*[c.ctypes.data for c in cells])
    arr, nl = _leaves(names, tpl.where, coltypes)
    threads = threads or os.cpu_count() or 1
    cap = 4096
    keys = np.zeros(2 * cap, np.int64)
    ints = np.zeros(3 * cap, np.int64)
    flts = np.zeros(3 * cap, np.float64)
    ng = C.c_uint64()
    ix = names.index
    sec = fn(ptrs, cells[0].shape[0], arr, nl, ix("flag_a"), ix("flag_b"), ix("quantity"), ix("price_cents"),
             ix("discount_pct"), ix("tax_pct"), threads, cap, keys.ctypes.data, ints.ctypes.data, flts.ctypes.data,
             C.byref(ng))
    g = min(int(ng.value), cap)
    rows = sorted((tuple(int(x) for x in keys[2 * i:2 * i + 2]), int(ints[3 * i]), int(ints[3 * i + 1]),
                   int(ints[3 * i + 2]), float(flts[3 * i]), float(flts[3 * i + 1]), float(flts[3 * i + 2]))
                  for i in range(g))
    return {"seconds": sec, "groups": rows, "threads": threads}


def highcard(cols: dict, threads: int | None = None, cap: int | None = None) -> dict:
    """GROUP BY key, count(*), sum(value) the reference's way (``ref_highcard``).
    Returns the wall seconds, the group count and (up to ``cap``) the groups
    as key-sorted arrays (keys, counts, sums)."""
    import os
    lib = load()
    fn = lib.ref_highcard
    fn.restype = C.c_double
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.POINTER(C.c_uint64)]
    key = np.ascontiguousarray(to_cells(cols["key"]))
    val = np.ascontiguousarray(to_cells(cols["value"]))
    threads = threads or os.cpu_count() or 1
    n = key.shape[0]
    cap = n if cap is None else cap
    k = np.zeros(max(1, cap), np.int64)
    c = np.zeros(max(1, cap), np.int64)
    s = np.zeros(max(1, cap), np.int64)
    ng = C.c_uint64()
    sec = fn(key.ctypes.data, val.ctypes.data, n, threads, cap, k.ctypes.data, c.ctypes.data, s.ctypes.data,
             C.byref(ng))
    g = min(int(ng.value), cap)
    order = np.argsort(k[:g], kind="stable")
    return {"seconds": sec, "ngroups": int(ng.value), "keys": k[:g][order], "counts": c[:g][order],
            "sums": s[:g][order], "threads": threads}


def join_group(fact: dict, dim: dict, day_lt: int, threads: int | None = None) -> dict:
    """The join + GROUP BY segment aggregate (sum(price*(100-disc)), count) the
    reference's way (``ref_join_group``). Returns the wall seconds and the
    groups sorted by segment: (segment, count, f64 sum)."""
    import os
    lib = load()
    fn = lib.ref_join_group
    fn.restype = C.c_double
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                   C.c_uint64, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]
    f = {k: np.ascontiguousarray(to_cells(fact[k])) for k in ("fk", "price_cents", "discount_pct")}
    d = {k: np.ascontiguousarray(to_cells(dim[k])) for k in ("key", "order_day", "segment")}
    threads = threads or os.cpu_count() or 1
    cap = 1024
    keys, counts, sums = np.zeros(cap, np.int64), np.zeros(cap, np.int64), np.zeros(cap, np.float64)
    ng = C.c_uint64()
    sec = fn(f["fk"].ctypes.data, f["price_cents"].ctypes.data, f["discount_pct"].ctypes.data, f["fk"].shape[0],
             d["key"].ctypes.data, d["order_day"].ctypes.data, d["segment"].ctypes.data, d["key"].shape[0],
             int(day_lt), threads, cap, keys.ctypes.data, counts.ctypes.data, sums.ctypes.data, C.byref(ng))
    g = min(int(ng.value), cap)
    rows = sorted((int(keys[i]), int(counts[i]), float(sums[i])) for i in range(g))
    return {"seconds": sec, "groups": rows, "threads": threads}
