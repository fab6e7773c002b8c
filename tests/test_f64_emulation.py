"""The reference's f64 aggregate arithmetic, emulated (oracle/f64_emulation.py):
where it equals the exact int128 oracle and where it does not."""
import math

import numpy as np

import oracle
from oracle import f64_emulation as F
from oracle import refpath
from turbogp_b200 import datagen, workloads

CT = datagen.LINEITEM_COLTYPES


def _loop_sum(e, cols, rows):
    """The per-shape rules as a plain row loop (small inputs only)."""
    def cell(name, r):
        return float(int(cols[name][r]) & 0xFFFFFFFFFFFFFFFF)

    def ev(x, r):
        if x[0] == "col":
            v = int(cols[x[1]][r])
        elif x[0] == "lit":
            v = x[1]
        else:
            a, b = ev(x[1], r), ev(x[2], r)
            v = {"mul": a * b, "sub": a - b, "add": a + b}[x[0]]
        v &= 0xFFFFFFFFFFFFFFFF
        return v - (1 << 64) if v >> 63 else v

    if e[0] == "col":
        s = 0
        for r in rows:
            s += ev(e, r)
        s &= 0xFFFFFFFFFFFFFFFF
        return s - (1 << 64) if s >> 63 else s
    s = 0.0
    l, rt = (e[1], e[2]) if len(e) == 3 else (None, None)
    for r in rows:
        if e[0] == "mul" and l[0] == "col" and rt[0] == "col":
            t = cell(l[1], r) * cell(rt[1], r)
        elif e[0] == "mul" and l[0] == "col":
            t = cell(l[1], r) * float(ev(rt, r))
        elif e[0] == "mul" and rt[0] == "col":
            t = float(ev(l, r)) * cell(rt[1], r)
        elif e[0] == "sub" and rt[0] == "col" and l[0] != "col":
            t = float(ev(l, r)) - cell(rt[1], r)
        elif e[0] == "sub" and l[0] == "col" and rt[0] != "col":
            t = cell(l[1], r) - float(ev(rt, r))
        elif e[0] == "add" and l[0] == "col" and rt[0] == "col":
            t = cell(l[1], r) + cell(rt[1], r)
        else:
            t = float(ev(e, r))
        s += t
    return s


def test_emulation_matches_a_row_loop():
    rng = np.random.default_rng(3)
    n = 3000
    cols = {"a": rng.integers(-10**6, 10**6, n).astype(np.int32),
            "b": rng.integers(0, 10**12, n).astype(np.int64),
            "g": rng.integers(0, 4, n).astype(np.uint8)}
    cols["a"][:3] = [-(2**31), 2**31 - 1, -1]   # negative cells are read as u64 words
    sel = np.flatnonzero(rng.random(n) < 0.7)
    c, k, mul, sub, add = F.c, F.k, F.mul, F.sub, F.add
    exprs = [c("a"), c("b"), mul(c("a"), c("b")), mul(c("b"), sub(k(100), c("a"))), mul(sub(k(7), c("a")), c("b")),
             mul(c("a"), k(3)), mul(k(-5), c("b")), sub(k(100), c("a")), sub(c("b"), mul(c("a"), k(2))),
             sub(c("b"), k(9)), add(c("a"), c("b")), mul(mul(c("b"), sub(k(100), c("a"))), add(k(100), c("a"))),
             k(11)]
    keys, counts, sums, _ = F.grouped(cols, sel, ("g",), exprs)
    for gi, key in enumerate(keys):
        rows = [int(r) for r in sel if int(cols["g"][r]) == key[0]]
        assert counts[gi] == len(rows)
        for e, s in zip(exprs, sums):
            want = _loop_sum(e, cols, rows)
            assert s[gi] == want and type(s[gi]) is type(want), (e, key)


def _exact(out):
    return {tuple(k): [v.value for v in vals] for k, vals in zip(out.keys, out.values)}


def test_grouped_aggregate_6m_where_the_reference_is_inexact():
    """6M-row filtered grouped aggregate: the reference's f64 sums equal the
    exact ones except sum(price*(100-disc)*(100+tax)), whose per-group sums
    (~5e16) pass 2^53."""
    n = 6_000_000
    host = datagen.lineitem(n, seed=1)
    tpl = workloads.filtered_group_agg()
    exact = oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where)
    sel = oracle.filter(host, CT, tpl.where).rowids.astype(np.int64)
    c, k, mul, sub, add = F.c, F.k, F.mul, F.sub, F.add
    disc_price = mul(c("price_cents"), sub(k(100), c("discount_pct")))
    charge = mul(disc_price, add(k(100), c("tax_pct")))
    keys, counts, sums, avgs = F.grouped(host, sel, tpl.group_by,
                                         [c("quantity"), c("price_cents"), disc_price, charge], [c("quantity")])
    ex = _exact(exact)
    assert sorted(ex) == keys
    inexact = 0
    for gi, key in enumerate(keys):
        cnt, s_qty, s_price, s_dp, s_ch, a_qty = ex[key]
        assert counts[gi] == cnt
        assert sums[0][gi] == s_qty and sums[1][gi] == s_price        # wrapping i64: exact
        assert sums[2][gi] == float(s_dp) and s_dp < 2**53             # f64, below 2^53: exact
        assert avgs[0][gi] == float(s_qty) / cnt
        emu = sums[3][gi]
        assert s_ch > 2**53
        # Sequential f64 summation: |error| <= (n - 1) * 2^-53 * sum |terms|.
        assert abs(emu - s_ch) <= (cnt - 1) * 2.0**-53 * s_ch
        inexact += emu != float(s_ch)
    assert inexact > 0   # the reference's sum_charge is not the exact sum
    # How far off: a few ulps of the result, far inside the bound above.
    worst = max(abs(sums[3][gi] - ex[key][4]) / math.ulp(float(ex[key][4])) for gi, key in enumerate(keys))
    assert worst < 1e4


def test_selective_scan_sum_matches_the_reference_path():
    """SUM(price * discount) as the reference sums it (u64 cells to f64, f64
    products, f64 sum in row order) equals ref_path.cpp and the exact sum."""
    n = 2_000_000
    host = datagen.lineitem(n, seed=2)
    cols = {k: host[k] for k in ("ship_day", "discount_pct", "quantity", "price_cents")}
    tpl = workloads.selective_scan_sum()
    sel = oracle.filter(host, CT, tpl.where).rowids.astype(np.int64)
    _, counts, sums, _ = F.grouped(host, sel, (), [F.mul(F.c("price_cents"), F.c("discount_pct"))])
    ref = refpath.selective_scan_sum(cols, tpl)
    exact = oracle.aggregate(host, CT, tpl.aggs, (), tpl.where)
    assert counts[0] == ref["count"] == exact.values[0][1].value
    assert sums[0][0] == ref["sum"] == float(exact.values[0][0].value)
