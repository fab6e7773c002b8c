"""The benchmark workloads at their full sizes on the GPU, with the inputs the
benchmark uses (same generators and seeds), against exact checkers:

* filtered grouped aggregate: 6M rows, against the row-at-a-time oracle and
  the numpy checker;
* join + grouped aggregate: 60M-row Zipf(0.8) fact table x 1.5M-row
  dimension, against the numpy checker;
* high-cardinality GROUP BY key: 100M rows, Zipf(1.1) over 10M keys, the
  benchmark's group capacity (10M), every group against numpy bincounts, and
  its ORDER BY count DESC LIMIT 10 form;
* a batch of 256 uneven queries over prefix views of the 60M-row table
  (the batching workload), each result equal to the same query run alone,
  and a sample of them against the numpy checker.

The numpy checker (oracle/scale.py) is pinned against the row-at-a-time
oracle by tests/test_scale_oracle.py."""
import numpy as np
import pytest

import oracle
from oracle import scale
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import col, count_star, sum_

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES
FCT = {**CT, "fk": "int"}


def same_query(a, b):
    assert a.rows_selected == b.rows_selected
    assert a.keys == b.keys
    assert len(a.values) == len(b.values)
    for ga, gb in zip(a.values, b.values):
        for x, y in zip(ga, gb):
            assert x.count == y.count
            assert x.value == y.value
            assert x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)


@pytest.fixture(scope="module")
def fact60():
    return datagen.fact_fk(60_000_000, 1_500_000, 0.8, seed=3)


@pytest.fixture(scope="module")
def dim15():
    return datagen.dimension(1_500_000, seed=2)


def test_filtered_group_agg_6m(ctx):
    host = datagen.lineitem(6_000_000, seed=1)
    t = ctx.register(host, CT)
    tpl = workloads.filtered_group_agg()
    g = t.prepare(tpl.aggs, tpl.group_by, tpl.where).run()
    same_query(g, oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where))
    same_query(g, scale.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where))
    assert len(g.keys) == 6
    t.drop()


def test_join_group_agg_60m_x_1_5m(ctx, fact60, dim15):
    fact = {k: fact60[k] for k in ("fk", "price_cents", "discount_pct", "quantity")}
    fct = {k: FCT[k] for k in fact}
    d = ctx.register(dim15, datagen.DIMENSION_COLTYPES)
    f = ctx.register(fact, fct)
    tpl = workloads.join_group_agg()
    j = d.join_build("key", tpl.build_where)
    build = (dim15, datagen.DIMENSION_COLTYPES, "key", tpl.build_where)
    for where in (None, col("quantity") < 24):
        g = f.aggregate(tpl.aggs, tpl.group_by, where, join=j, probe_key="fk")
        e = scale.aggregate(fact, fct, tpl.aggs, tpl.group_by, where, build=build, probe_key="fk")
        same_query(g, e)
        assert len(g.keys) == 25
    j.drop()
    f.drop()
    d.drop()


def test_highcard_group_100m(ctx):
    host = datagen.highcard(100_000_000, 10_000_000, 1.1, seed=4)
    t = ctx.register(host)
    aggs = [count_star(), sum_(col("value"))]
    q = t.prepare(aggs, ("key",), None, group_cap=10_000_000)
    out = q.run()
    keys, lo, hi, cnt = out.arrays()
    ek, ec, es = scale.group_count_sum(host["key"], host["value"])
    assert out.rows_selected == 100_000_000
    assert keys.shape[0] == ek.shape[0]
    assert np.array_equal(keys[:, 0], ek)
    assert np.array_equal(lo[:, 0].view(np.int64), ec) and not hi[:, 0].any()
    assert np.array_equal(lo[:, 1].view(np.int64), es) and not hi[:, 1].any()
    assert np.array_equal(cnt[:, 0].view(np.int64), ec) and np.array_equal(cnt[:, 1].view(np.int64), ec)
    # ORDER BY count(*) DESC LIMIT 10: the ten largest counts, ties by key.
    top = t.aggregate_topn(aggs, ("key",), None, 0, True, 10)
    order = np.lexsort((ek, -ec))[:10]
    assert [k[0] for k in top.keys] == ek[order].tolist()
    assert [r[0].value for r in top.values] == ec[order].tolist()
    assert [r[1].value for r in top.values] == es[order].tolist()
    t.drop()


def test_batch_of_256_uneven_queries_at_full_size(ctx, fact60, dim15):
    import torch
    from bench import batch_queries
    fact = {k: torch.from_numpy(v).to("cuda:0") for k, v in fact60.items()}
    pqs, rows, _, keep = batch_queries(ctx, fact, dim15, 256, seed=11)
    batched = ctx.submit(pqs).wait()
    alone = [q.run() for q in pqs]
    for b, a in zip(batched, alone):
        same_query(b, a)
    # A sample against the exact checker: the smallest and largest views of
    # every template (template = query shape), on the host data.
    tj = workloads.join_group_agg()
    build = (dim15, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
    picked = {}
    for i, pq in enumerate(pqs):
        shape = (pq.nk, pq.na, int(pq.q.join != 0))
        lo, hi = picked.get(shape, (i, i))
        picked[shape] = (lo if rows[lo] <= rows[i] else i, hi if rows[hi] >= rows[i] else i)
    for i in sorted({i for pair in picked.values() for i in pair}):
        pq = pqs[i]
        view = {k: v[:rows[i]] for k, v in fact60.items()}
        spec = pq.spec
        e = scale.aggregate(view, FCT, spec["aggs"], spec["group_by"], spec["where"],
                            build=build if spec["join"] else None, probe_key="fk" if spec["join"] else None)
        same_query(batched[i], e)
    del keep
