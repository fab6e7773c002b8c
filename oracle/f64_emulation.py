"""TEST INFRASTRUCTURE: the reference's f64 aggregate sums, emulated.

The exact oracle (``oracle.cpp``) sums in int128. The reference sums most
integer aggregate arguments in f64 instead, so where partial sums pass 2^53 its
results are not exact; this module reproduces its arithmetic to document where.

What the reference computes for SUM(e) over a group (``sum_vec``,
src/engine/query_interpreter/aggregate.rs:1485-1792, integer columns):

* ``SUM(col)``: a wrapping i64 sum (1499-1504), exact unless it wraps.
* ``SUM(a * b)``, both plain columns: ``a as f64 * b as f64`` per row, where the
  cells are the u64 words of the table (1598-1601), then an f64 sum.
* ``SUM(a * e)`` / ``SUM(e * b)`` with one plain column and an expression
  holding columns: ``cell as f64 * eval(e) as f64`` per row (1606-1616,
  1642-1655); with a constant instead: ``cell as f64 * f64(constant)``.
* ``SUM(k - b)``, ``SUM(a - e)``, ``SUM(a - k)`` and ``SUM(a + b)``: the same
  per-row f64 forms (1685-1760).
* anything else: the row's exact wrapping-i64 value (``binop``,
  expr.rs:2063-2076) converted to f64, then an f64 sum (1672-1680, 1781-1789).

Terms are added one by one in ascending row order within each group: the group
row lists are built per 65,536-row chunk and merged in chunk order
(aggregate.rs:580-623). AVG is the f64 of that sum divided by the row count
(aggregate.rs:1416-1424).

Expressions are small tuples: ``("col", name)``, ``("lit", k)``,
``("mul" | "sub" | "add", left, right)``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def c(name: str) -> tuple:
    return ("col", name)


def k(v: int) -> tuple:
    return ("lit", int(v))


def mul(a, b) -> tuple:
    return ("mul", a, b)


def sub(a, b) -> tuple:
    return ("sub", a, b)


def add(a, b) -> tuple:
    return ("add", a, b)


def _has_col(e) -> bool:
    return e[0] == "col" or (e[0] in ("mul", "sub", "add") and (_has_col(e[1]) or _has_col(e[2])))


def _eval_i64(e, cols: dict, sel: np.ndarray) -> np.ndarray:
    """The row's value as the reference's ``eval`` computes it: wrapping i64."""
    with np.errstate(over="ignore"):
        if e[0] == "col":
            return cols[e[1]][sel].astype(np.int64)
        if e[0] == "lit":
            return np.full(sel.shape[0], e[1], dtype=np.int64)
        a, b = _eval_i64(e[1], cols, sel), _eval_i64(e[2], cols, sel)
        return {"mul": np.multiply, "sub": np.subtract, "add": np.add}[e[0]](a, b)


def _const(e) -> float:
    assert not _has_col(e)
    return float(_eval_i64(e, {}, np.zeros(1, dtype=np.int64))[0])


def _cell_f64(e, cols: dict, sel: np.ndarray) -> np.ndarray:
    """``cell as f64`` of a plain integer column: the u64 word, unsigned."""
    return cols[e[1]][sel].astype(np.int64).view(np.uint64).astype(np.float64)


def sum_terms(e, cols: dict, sel: np.ndarray) -> tuple[str, np.ndarray]:
    """Per-row terms of the reference's SUM(e) over the rows ``sel``:
    ("i64", terms) for a wrapping integer sum, ("f64", terms) for an f64 sum."""
    op = e[0]
    if op == "col":
        return "i64", _eval_i64(e, cols, sel)
    if op in ("mul", "sub", "add"):
        l, r = e[1], e[2]
        lc, rc = l[0] == "col", r[0] == "col"
        if op == "mul":
            if lc and rc:
                return "f64", _cell_f64(l, cols, sel) * _cell_f64(r, cols, sel)
            if lc:
                rf = _eval_i64(r, cols, sel).astype(np.float64) if _has_col(r) else _const(r)
                return "f64", _cell_f64(l, cols, sel) * rf
            if rc:
                lf = _eval_i64(l, cols, sel).astype(np.float64) if _has_col(l) else _const(l)
                return "f64", lf * _cell_f64(r, cols, sel)
        elif op == "sub":
            if not lc and rc:
                if _has_col(l):
                    raise NotImplementedError("the reference evaluates the left side as a constant here")
                return "f64", _const(l) - _cell_f64(r, cols, sel)
            if lc and not rc:
                rf = _eval_i64(r, cols, sel).astype(np.float64) if _has_col(r) else _const(r)
                return "f64", _cell_f64(l, cols, sel) - rf
        elif lc and rc:
            return "f64", _cell_f64(l, cols, sel) + _cell_f64(r, cols, sel)
    return "f64", _eval_i64(e, cols, sel).astype(np.float64)


def grouped(columns: dict, sel: np.ndarray, group_by=(), sums=(), avgs=()):
    """The reference's SUM / AVG values per group over the selected rows
    ``sel`` (ascending row ids). Groups are exact key tuples in ascending
    order. Returns (keys, counts, sums, avgs): a list of key tuples, the row
    count per group, one list per SUM expression (int for a wrapping i64 sum,
    float for an f64 sum) and one list of floats per AVG expression."""
    sel = np.asarray(sel, dtype=np.int64)
    if group_by:
        keys = np.stack([columns[g][sel].astype(np.int64) for g in group_by], axis=1)
        uniq, gid = np.unique(keys, axis=0, return_inverse=True)
        gid = gid.reshape(-1).astype(np.uint32)
        key_list = [tuple(int(x) for x in row) for row in uniq]
    else:
        gid = np.zeros(sel.shape[0], dtype=np.uint32)
        key_list = [()]
    ng = len(key_list)
    counts = np.bincount(gid, minlength=ng).astype(np.int64)

    def one(e):
        kind, terms = sum_terms(e, columns, sel)
        if kind == "i64":
            acc = np.zeros(ng, dtype=np.int64)
            with np.errstate(over="ignore"):
                np.add.at(acc, gid, terms)
            return [int(x) for x in acc]
        terms = np.ascontiguousarray(terms, dtype=np.float64)
        out = np.zeros(ng, dtype=np.float64)
        _lib().orc_seq_sum_f64(terms.ctypes.data, np.ascontiguousarray(gid).ctypes.data, C.c_uint64(terms.shape[0]),
                               C.c_uint32(ng), out.ctypes.data)
        return [float(x) for x in out]

    sum_vals = [one(e) for e in sums]
    avg_vals = []
    for e in avgs:
        s = one(e)
        avg_vals.append([float(x) / float(n) if n else 0.0 for x, n in zip(s, counts)])
    return key_list, [int(x) for x in counts], sum_vals, avg_vals
