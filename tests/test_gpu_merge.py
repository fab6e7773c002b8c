"""Merged scans inside a batch (tgp_batch_submit): queries of one shape whose
WHERE literals differ on one column run as a single scan grouped by that
column's buckets, and every query's result — groups, exact sums, counts,
MIN / MAX, rows_selected — equals the query run alone and the oracle's.
Cases: range, equality, <> and NOT BETWEEN literals (buckets that are not
intervals), identical queries, empty and full selections, a common extra
leaf, MIN / MAX values, joins (whose rows_selected needs per-bucket counts),
a class larger than 64 queries (split into several merged scans), and
scan queries whose literals differ on three columns (one bucket key per
column; a member accepts a combination of buckets when it accepts each)."""
import numpy as np
import pytest

import oracle
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import avg, build_col, col, count_col, count_star, max_, min_, sum_

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES
FCT = {**CT, "fk": "int"}
D0, ND = datagen.DAY0, datagen.NDAYS


def same_query(a, b):
    assert a.rows_selected == b.rows_selected and a.keys == b.keys
    for ra, rb in zip(a.values, b.values):
        for x, y in zip(ra, rb):
            assert (x.value, x.count) == (y.value, y.count)
            assert x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)


def test_merged_batches_equal_queries_alone(ctx):
    rng = np.random.default_rng(101)
    fact = datagen.fact_fk(1_500_007, 30_000, 0.8, seed=102)
    dim = datagen.dimension(30_000, seed=103)
    f = ctx.register(fact, FCT)
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    tj = workloads.join_group_agg()
    j = d.join_build("key", tj.build_where)
    fga = workloads.filtered_group_agg()
    q = col("quantity")
    mm_aggs = [count_star(), min_(col("price_cents")), max_(col("discount_pct") * 3), sum_(q), count_col(col("tax_pct"))]
    specs = []   # (aggs, group_by, where, join)
    for x in list(rng.integers(D0 - 5, D0 + ND + 5, 70)) + [D0 + 100, D0 + 100, D0 - 1]:
        specs.append((fga.aggs, fga.group_by, col("ship_day") <= int(x), None))
    for x in rng.integers(D0, D0 + ND, 6):
        specs.append((fga.aggs, fga.group_by, (col("tax_pct") < 5) & (col("ship_day") > int(x)), None))
    for c in list(rng.integers(0, 52, 20)) + [0, 100]:
        specs.append((tj.aggs, tj.group_by, q < int(c), j))
    for a, b in rng.integers(0, 52, (8, 2)):
        lo, hi = int(min(a, b)), int(max(a, b))
        specs.append((mm_aggs, ("flag_a",), q.between(lo, hi), None))
        specs.append((mm_aggs, ("flag_a",), q.not_between(lo, hi), None))
        specs.append((mm_aggs, ("flag_a",), q != lo, None))
    for c in rng.integers(1, 50, 6):
        specs.append(([count_star(), sum_(col("price_cents") * build_col("segment"))], (build_col("segment"), "flag_b"),
                      q >= int(c), j))
    for _ in range(40):
        tpl = workloads.selective_scan_sum(day_lo=D0 + int(rng.integers(0, 2000)), days=int(rng.integers(30, 526)),
                                           disc_lo=int(rng.integers(0, 6)), disc_hi=int(rng.integers(5, 11)),
                                           qty_lt=int(rng.integers(2, 51)))
        specs.append((tpl.aggs, tpl.group_by, tpl.where, None))
    pqs = [f.prepare(a, g, w, join=jj, probe_key="fk" if jj else None) for a, g, w, jj in specs]
    order = rng.permutation(len(pqs))
    batch = [pqs[i] for i in order]
    outs = ctx.submit(batch).wait()
    alone = [pq.run() for pq in batch]
    for o, a in zip(outs, alone):
        same_query(o, a)
    # A sample against the oracle.
    build = (dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
    for k in range(0, len(batch), 7):
        a, g, w, jj = specs[order[k]]
        e = oracle.aggregate(fact, FCT, a, g, w, build=build if jj else None, probe_key="fk" if jj else None)
        same_query(outs[k], e)
    # The same batch again (plans, buffers and merged scans reused), polled.
    h = ctx.submit(batch)
    while not h.poll():
        pass
    for o, a in zip(h.wait(), alone):
        same_query(o, a)
    j.drop()
    f.drop()
    d.drop()


def test_batch_mixing_join_group_layouts(ctx):
    """One batch over one join whose queries fold different build-side group
    layouts into payload arrays: a lone join query (25 groups), a merged class
    of join queries (quantity buckets x 25 groups) and joins grouped by
    (segment, order_day) and by order_day alone. Each layout keeps its own
    payload array, so every result equals the query run alone and the
    oracle's, in either submission order."""
    rng = np.random.default_rng(7)
    fact = datagen.fact_fk(700_003, 20_000, 0.8, seed=71)
    dim = datagen.dimension(20_000, seed=72)
    f = ctx.register(fact, FCT)
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    tj = workloads.join_group_agg()
    j = d.join_build("key", tj.build_where)
    q = col("quantity")
    specs = [([count_star()], tj.group_by, q < 30)]
    specs += [(tj.aggs, tj.group_by, q < int(c)) for c in rng.integers(1, 52, 24)]
    specs += [([count_star(), sum_(col("price_cents"))], (build_col("segment"), build_col("order_day")), q < 40),
              ([sum_(q), count_star()], (build_col("order_day"),), None)]
    pqs = [f.prepare(a, g, w, join=j, probe_key="fk") for a, g, w in specs]
    build = (dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
    for batch_order in (list(range(len(pqs))), list(range(len(pqs)))[::-1]):
        batch = [pqs[i] for i in batch_order]
        outs = ctx.submit(batch).wait()
        for i, o in zip(batch_order, outs):
            same_query(o, pqs[i].run())
            if i in (0, 1, len(pqs) - 2, len(pqs) - 1):
                a, g, w = specs[i]
                same_query(o, oracle.aggregate(fact, FCT, a, g, w, build=build, probe_key="fk"))
    j.drop()
    f.drop()
    d.drop()
