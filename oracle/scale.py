"""TEST INFRASTRUCTURE: exact numpy checkers for the benchmark workloads at
their full sizes (6M, 60M x 1.5M, 100M rows), where the row-at-a-time oracle
(``oracle.cpp``) would take minutes.

The semantics are the oracle's, which restates the reference's:

* predicate leaves compare the u64 cell of a value: Int columns as signed i64,
  Date columns as unsigned, ``=`` / ``<>`` bitwise
  (src/engine/query_interpreter/expr.rs:1468-1530, src/exec/bitmap.rs:321-480);
  BETWEEN = ge AND le, NOT BETWEEN = lt OR gt (expr.rs:687-760); AND / OR /
  NOT over the row masks (expr.rs:633-679);
* a per-row aggregate argument is the product of affine factors ``mul * cell +
  add`` in i64 (expr.rs:2063-2076; a wrap raises here instead of wrapping, the
  workloads never wrap);
* SUM is exact (the reference accumulates f64, aggregate.rs:1605-1622); COUNT
  counts rows; COUNT(col) counts nonzero arguments (accum_grouped.rs:243-246);
  AVG carries the exact sum and the row count;
* groups are exact key tuples in ascending order; the inner equi-join matches
  each probe row with the build rows of equal key that pass the build filter
  (join.rs:544-794); the build keys must be unique here (the row-at-a-time
  oracle covers duplicate keys at small sizes).

Exact sums: each i64 argument is split into three 24-bit limbs whose per-group
sums stay below 2^53 (for fewer than 2^29 rows), summed with float64
``bincount`` and recombined as Python integers.

Only ``tests/`` and ``bench.py``'s CPU-baseline leg use this module, as a
checker. ``tests/test_scale_oracle.py`` pins it against ``oracle.aggregate``.
"""
from __future__ import annotations

import numpy as np

from turbogp_b200 import _capi as A
from turbogp_b200.engine import AggResult, Col, QueryOutput

_MASK64 = (1 << 64) - 1


def _cells(a: np.ndarray) -> np.ndarray:
    """The reference's u64 cell of each value, as int64 bits (u8 zero-extended,
    i32 sign-extended, 64-bit as stored)."""
    if a.dtype == np.uint8:
        return a.astype(np.int64)
    if a.dtype == np.int32:
        return a.astype(np.int64)
    return a.view(np.int64)


def _lit(v: int) -> int:
    """A literal as the signed i64 of its 64-bit pattern."""
    v = int(v) & _MASK64
    return v - (1 << 64) if v >> 63 else v


def _leaf(cells: np.ndarray, coltype: str, cmp: int, lit: int, lit2: int) -> np.ndarray:
    if coltype == "float":
        raise NotImplementedError("FLOAT leaves are checked by the row-at-a-time oracle")
    if cmp in (A.CMP_EQ, A.CMP_NE):
        m = cells == _lit(lit)
        return m if cmp == A.CMP_EQ else ~m
    x = cells if coltype == "int" else cells.view(np.uint64)
    cv = (lambda v: np.int64(_lit(v))) if coltype == "int" else (lambda v: np.uint64(int(v) & _MASK64))
    a, b = cv(lit), cv(lit2)
    if cmp == A.CMP_LT:
        return x < a
    if cmp == A.CMP_LE:
        return x <= a
    if cmp == A.CMP_GT:
        return x > a
    if cmp == A.CMP_GE:
        return x >= a
    if cmp == A.CMP_BETWEEN:
        return (x >= a) & (x <= b)
    if cmp == A.CMP_NOT_BETWEEN:
        return (x < a) | (x > b)
    raise ValueError(f"comparison {cmp}")


def where_mask(columns: dict, coltypes: dict | None, where, n: int) -> np.ndarray:
    """Row mask of a WHERE tree (a Pred in postfix form, or None = all rows)."""
    coltypes = coltypes or {}
    if where is None or not where.ops:
        return np.ones(n, dtype=bool)
    stack: list[np.ndarray] = []
    for op in where.ops:
        if op[0] == "leaf":
            _, name, cmp, v, v2 = op
            stack.append(_leaf(_cells(columns[name]), coltypes.get(name, "int"), cmp, v, v2))
        elif op[0] == "not":
            stack.append(~stack.pop())
        else:
            b, a = stack.pop(), stack.pop()
            stack.append(a & b if op[0] == "and" else a | b)
    if len(stack) != 1:
        raise ValueError("malformed predicate program")
    return stack[0]


def _term(probe: dict, build: dict | None, brow: np.ndarray | None, sel: np.ndarray, term) -> np.ndarray:
    """The i64 argument of each selected row (sel: selected probe row ids)."""
    out = None
    big = None
    for f in term.factors:
        if f.column is None:
            x = np.full(sel.shape[0], f.add, dtype=np.int64)
        else:
            src = probe[f.column][sel] if f.side == A.SIDE_PROBE else build[f.column][brow]
            x = _cells(src) * np.int64(f.mul) + np.int64(f.add)
        xb = np.abs(x.astype(np.float64))
        out = x if out is None else out * x
        big = xb if big is None else big * xb
    if out is None:
        return np.ones(sel.shape[0], dtype=np.int64)
    if big.size and float(big.max()) >= 2.0 ** 62:
        raise OverflowError("a per-row argument leaves int64 (the workloads never do)")
    return out


def _group_sums(gid: np.ndarray, x: np.ndarray, ngroups: int) -> list[int]:
    """Exact per-group sums of int64 values (fewer than 2^29 rows)."""
    if x.shape[0] >= (1 << 29):
        raise ValueError("too many rows for the 24-bit limb sums")
    u = x.view(np.uint64)
    lo = (u & np.uint64(0xFFFFFF)).astype(np.float64)
    mid = ((u >> np.uint64(24)) & np.uint64(0xFFFFFF)).astype(np.float64)
    hi = (x >> np.int64(48)).astype(np.float64)  # signed top 16 bits
    s_lo = np.bincount(gid, weights=lo, minlength=ngroups)
    s_mid = np.bincount(gid, weights=mid, minlength=ngroups)
    s_hi = np.bincount(gid, weights=hi, minlength=ngroups)
    return [int(s_hi[g]) * (1 << 48) + int(s_mid[g]) * (1 << 24) + int(s_lo[g]) for g in range(ngroups)]


def _group_reduce(gid: np.ndarray, x: np.ndarray, ngroups: int, fn) -> list[int]:
    out = np.full(ngroups, np.iinfo(np.int64).max if fn is np.minimum else np.iinfo(np.int64).min, dtype=np.int64)
    fn.at(out, gid, x)
    return [int(v) for v in out]


def aggregate(columns: dict, coltypes: dict | None, aggs, group_by=(), where=None, build=None,
              probe_key: str | None = None) -> QueryOutput:
    """The exact result of a scalar / grouped aggregate (optionally over an
    inner join with ``build`` = (columns, coltypes, key name, where)), in the
    engine's QueryOutput shape: groups with at least one row, ascending keys."""
    n = next(iter(columns.values())).shape[0]
    sel = np.flatnonzero(where_mask(columns, coltypes, where, n))
    n_selected = int(sel.shape[0])  # rows passing the probe-side WHERE (before the join)
    bcols, brow = None, None
    if build is not None:
        bcols, bct, bkey, bwhere = build
        nb = next(iter(bcols.values())).shape[0]
        bsel = np.flatnonzero(where_mask(bcols, bct, bwhere, nb))
        bk = _cells(bcols[bkey])[bsel]
        if np.unique(bk).shape[0] != bk.shape[0]:
            raise NotImplementedError("duplicate build keys are checked by the row-at-a-time oracle")
        order = np.argsort(bk, kind="stable")
        bk_sorted, brow_sorted = bk[order], bsel[order]
        pk = _cells(columns[probe_key])[sel]
        pos = np.searchsorted(bk_sorted, pk)
        pos_c = np.minimum(pos, max(bk_sorted.shape[0] - 1, 0))
        hit = (pos < bk_sorted.shape[0]) & (bk_sorted[pos_c] == pk) if bk_sorted.shape[0] else np.zeros_like(pk, bool)
        sel = sel[hit]
        brow = brow_sorted[pos_c[hit]]
    # Group ids: dense over each key's [min, max] range when that is small,
    # else by sorting the key tuples.
    keys = []
    for g in group_by:
        c = g if isinstance(g, Col) else Col(g)
        src = columns[c.name][sel] if c.side == A.SIDE_PROBE else bcols[c.name][brow]
        keys.append(_cells(src))
    if not keys:
        gid = np.zeros(sel.shape[0], dtype=np.int64)
        ngroups, gkeys = 1, [()]
    else:
        los = [int(k.min()) if k.size else 0 for k in keys]
        spans = [int(k.max()) - lo + 1 if k.size else 1 for k, lo in zip(keys, los)]
        dom = 1
        for s in spans:
            dom *= s
        if dom <= 64 * max(sel.shape[0], 1) and dom <= (1 << 31):
            gid = np.zeros(sel.shape[0], dtype=np.int64)
            for k, lo, s in zip(keys, los, spans):
                gid = gid * s + (k - lo)
            present = np.bincount(gid, minlength=dom) > 0
            dense_ids = np.flatnonzero(present)
            remap = np.full(dom, -1, dtype=np.int64)
            remap[dense_ids] = np.arange(dense_ids.shape[0])
            gkeys = []
            for d in dense_ids.tolist():
                t = []
                for lo, s in zip(reversed(los), reversed(spans)):
                    t.append(lo + d % s)
                    d //= s
                gkeys.append(tuple(reversed(t)))
            gid = remap[gid]
            ngroups = dense_ids.shape[0]
        else:
            tup = np.stack(keys, axis=1)
            uniq, gid = np.unique(tup, axis=0, return_inverse=True)
            gid = gid.reshape(-1)
            gkeys = [tuple(int(v) for v in r) for r in uniq]
            ngroups = uniq.shape[0]
    counts = np.bincount(gid, minlength=ngroups).astype(np.int64).tolist() if sel.size else [0] * ngroups
    per_agg = []
    for a in aggs:
        if a.func == A.AGG_COUNT_STAR:
            per_agg.append(counts)
            continue
        x = _term(columns, bcols, brow, sel, a.term)
        if a.func in (A.AGG_SUM, A.AGG_AVG):
            per_agg.append(_group_sums(gid, x, ngroups))
        elif a.func == A.AGG_COUNT_NONZERO:
            per_agg.append(np.bincount(gid, weights=(x != 0).astype(np.float64), minlength=ngroups).astype(np.int64).tolist())
        elif a.func == A.AGG_MIN:
            per_agg.append(_group_reduce(gid, x, ngroups, np.minimum))
        elif a.func == A.AGG_MAX:
            per_agg.append(_group_reduce(gid, x, ngroups, np.maximum))
        else:
            raise ValueError(f"aggregate {a.func}")
    out_keys, out_vals = [], []
    for g in range(ngroups):
        if group_by and counts[g] == 0:
            continue
        row = []
        for a, vals in zip(aggs, per_agg):
            v = vals[g]
            c = counts[g]
            f = (float(v) / c if c else 0.0) if a.func == A.AGG_AVG else float(v)
            row.append(AggResult(v, c, f))
        out_keys.append(gkeys[g])
        out_vals.append(row)
    return QueryOutput(out_keys, out_vals, n, n_selected, 0)


def group_count_sum(keys: np.ndarray, values: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """GROUP BY one integer key: (ascending distinct keys, row counts, exact
    sums of the values) with no Python objects per group — for the
    high-cardinality workload's millions of groups (|sum| < 2^53 per group:
    checked)."""
    k = keys.astype(np.int64, copy=False)
    lo = int(k.min()) if k.size else 0
    span = int(k.max()) - lo + 1 if k.size else 1
    if span > (1 << 31):
        uniq, gid = np.unique(k, return_inverse=True)
        counts = np.bincount(gid, minlength=uniq.shape[0])
        sums = np.bincount(gid, weights=values.astype(np.float64), minlength=uniq.shape[0])
        present_keys = uniq
    else:
        rel = k - lo
        counts = np.bincount(rel, minlength=span)
        sums = np.bincount(rel, weights=values.astype(np.float64), minlength=span)
        present = np.flatnonzero(counts)
        present_keys, counts, sums = present + lo, counts[present], sums[present]
    if sums.size and float(np.abs(sums).max()) >= 2.0 ** 53:
        raise OverflowError("a group sum reaches 2^53: use aggregate() instead")
    return present_keys.astype(np.int64), counts.astype(np.int64), sums.astype(np.int64)
