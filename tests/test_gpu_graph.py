"""Captured queries (tgp_graph_capture / tgp_graph_launch): replays of one
graph against tgp_execute and the oracle, and the checks that refuse a graph
whose table or join changed under it."""
import numpy as np
import pytest

import oracle
from turbogp_b200 import _capi as A
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import avg, build_col, col, count_star, max_, min_, sum_

from test_gpu_parity import same_query

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES


def lineitem_queries():
    c = col
    s = workloads.selective_scan_sum()
    f = workloads.filtered_group_agg()
    return [
        (s.aggs, s.group_by, s.where),
        (f.aggs, f.group_by, f.where),
        ([count_star(), min_(c("price_cents")), max_(c("quantity") * c("tax_pct")), avg(c("discount_pct"))],
         ("flag_a",), c("quantity") < 17),
        ([sum_(c("price_cents") * (100 - c("discount_pct")))], (), c("flag_b") == 5),  # nothing passes
    ]


@pytest.mark.parametrize("n", [0, 1, 2049, 100_003])
def test_graph_replays_match_execute_and_oracle(ctx, n):
    host = datagen.lineitem(n, seed=31 + n)
    t = ctx.register(host, CT)
    for aggs, group_by, where in lineitem_queries():
        o = oracle.aggregate(host, CT, aggs, group_by, where)
        plain = t.prepare(aggs, group_by, where)
        same_query(plain.run(), o)
        g = t.prepare(aggs, group_by, where).capture()
        assert g.graph
        for _ in range(3):  # every replay clears its accumulators
            same_query(g.run(), o)
        g.drop_graph()
        same_query(g.run(), o)  # back on tgp_execute
    t.drop()


def test_graph_rebind_recaptures(ctx):
    host = datagen.lineitem(50_000, seed=5)
    t = ctx.register(host, CT)
    tpl = workloads.filtered_group_agg()
    g = t.prepare(tpl.aggs, tpl.group_by, tpl.where).capture()
    first = g.graph
    for d in [datagen.DAY0 + 100, datagen.DAY0 + 2000]:
        w = col("ship_day") <= d
        g.rebind(w)
        assert g.graph and g.graph != first
        same_query(g.run(), oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, w))
    t.drop()


def test_graph_join_aggregate(ctx):
    dim = datagen.dimension(40_000, seed=3)
    fact = datagen.fact_fk(300_000, 40_000, 0.8, seed=4)
    fact["fk"][:50] = 70_000  # keys beyond the build side
    fct = {**CT, "fk": "int"}
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    f = ctx.register(fact, fct)
    tpl = workloads.join_group_agg()
    j = d.join_build("key", tpl.build_where)
    for where in [None, col("quantity") < 30]:
        g = f.prepare(tpl.aggs, tpl.group_by, where, join=j, probe_key="fk").capture()
        o = oracle.aggregate(fact, fct, tpl.aggs, tpl.group_by, where,
                             build=(dim, datagen.DIMENSION_COLTYPES, "key", tpl.build_where), probe_key="fk")
        for _ in range(2):
            same_query(g.run(), o)
        g.drop_graph()
    # Queries of other build-side key layouts get payload arrays of their
    # own: the graph's array is not rewritten, so it still runs, exactly.
    g = f.prepare(tpl.aggs, tpl.group_by, None, join=j, probe_key="fk").capture()
    build = (dim, datagen.DIMENSION_COLTYPES, "key", tpl.build_where)
    for other in [(build_col("segment"), "flag_a"), (build_col("order_day"),)]:
        same_query(f.aggregate(tpl.aggs, other, None, join=j, probe_key="fk"),
                   oracle.aggregate(fact, fct, tpl.aggs, other, None, build=build, probe_key="fk"))
        same_query(g.run(), oracle.aggregate(fact, fct, tpl.aggs, tpl.group_by, None, build=build, probe_key="fk"))
    # A dropped join invalidates the graph.
    j.drop()
    with pytest.raises(A.TgpError) as e:
        g.run()
    assert e.value.status == A.NOT_FOUND
    g.drop_graph()


def test_graph_refuses_hash_grouping_and_changed_tables(ctx):
    rng = np.random.default_rng(6)
    h = {"key": rng.integers(0, 2**40, 20_000, dtype=np.int64),  # key range far above direct indexing
         "value": rng.integers(0, 1001, 20_000, dtype=np.int32)}
    th = ctx.register(h)
    with pytest.raises(A.TgpError) as e:
        th.prepare([count_star(), sum_(col("value"))], ("key",), None, group_cap=20_000).capture()
    assert e.value.status == A.UNSUPPORTED

    host = datagen.lineitem(30_000, seed=8)
    t = ctx.register(host, CT)
    tpl = workloads.filtered_group_agg()
    g = t.prepare(tpl.aggs, tpl.group_by, tpl.where).capture()
    same_query(g.run(), oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where))

    # Reload with new rows but the same min / max of every column: the graph
    # stays valid and sees the new rows.
    new = {k: v.copy() for k, v in host.items()}
    for k in new:
        rng.shuffle(new[k])  # each column's multiset, hence its min / max, is unchanged
    t.reload(new)
    same_query(g.run(), oracle.aggregate(new, CT, tpl.aggs, tpl.group_by, tpl.where))

    # A reload that moves a column's max refuses the graph (its bounds were
    # proven from the old statistics); a fresh capture runs.
    new2 = {k: v.copy() for k, v in host.items()}
    new2["price_cents"][7] = int(new2["price_cents"].max()) + 1
    t.reload(new2)
    with pytest.raises(A.TgpError) as e:
        g.run()
    assert e.value.status == A.NOT_FOUND
    g.capture()
    same_query(g.run(), oracle.aggregate(new2, CT, tpl.aggs, tpl.group_by, tpl.where))

    # A dropped table refuses it as well.
    t.drop()
    with pytest.raises(A.TgpError) as e:
        g.run()
    assert e.value.status == A.NOT_FOUND
    g.drop_graph()
    with pytest.raises(A.TgpError) as e:
        ctx._check(ctx.lib.tgp_graph_drop(ctx.h, 123456789), "tgp_graph_drop")
    assert e.value.status == A.NOT_FOUND
