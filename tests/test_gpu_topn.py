"""tgp_execute_topn: ORDER BY one aggregate LIMIT n, on hash-grouped (device
ordering) and direct-indexed (host ordering) results, against the oracle's
full result ordered by exact value with ties in ascending key order."""
import numpy as np
import pytest

import oracle
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import avg, col, count_star, max_, min_, sum_

from test_gpu_parity import same_query

pytestmark = pytest.mark.gpu


def expected(full, agg: int, desc: bool, limit: int, by_f64: bool):
    """The oracle's groups (ascending key order) sorted stably by the
    aggregate, so ties keep ascending key order, then cut at ``limit``."""
    keyf = (lambda i: full.values[i][agg].as_f64) if by_f64 else (lambda i: full.values[i][agg].value)
    order = sorted(range(len(full.keys)), key=keyf, reverse=desc)[:limit]

    class R:
        pass
    r = R()
    r.keys = [full.keys[i] for i in order]
    r.values = [full.values[i] for i in order]
    r.rows_selected = full.rows_selected
    return r


def check(g, e):
    assert g.keys == e.keys
    same_query(g, e)


@pytest.mark.parametrize("n", [1, 5000, 300_000])
def test_topn_hash_groups(ctx, n):
    rng = np.random.default_rng(n)
    ranks = datagen.zipf_ranks(n, 50_000, 1.1, rng)
    key = (ranks * 7_919_993).astype(np.int64) - 2**35     # sparse, signed keys: hash grouping
    cols = {"key": key, "v": rng.integers(-1000, 1001, n).astype(np.int32),
            "w": rng.integers(0, 2**62, n, dtype=np.int64)}  # sum(w) has no int64 bound: int128 ordering
    t = ctx.register(cols)
    aggs = [count_star(), sum_(col("v")), avg(col("v")), min_(col("v")), max_(col("w")), sum_(col("w"))]
    where = col("v") != 7
    full = oracle.aggregate(cols, None, aggs, ("key",), where)
    for agg, by_f64 in [(0, False), (1, False), (2, True), (3, False), (4, False), (5, False)]:
        for desc in (True, False):
            for limit in (1, 10, 1000, 10**6):
                g = t.aggregate_topn(aggs, ("key",), where, agg, desc, limit)
                check(g, expected(full, agg, desc, limit, by_f64))
    assert len(t.aggregate_topn(aggs, ("key",), where, 0, True, 0).keys) == 0
    t.drop()


def test_topn_direct_groups_and_scalar(ctx):
    host = datagen.lineitem(200_000, seed=9)
    CT = datagen.LINEITEM_COLTYPES
    t = ctx.register(host, CT)
    tpl = workloads.filtered_group_agg()
    full = oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where)
    for agg, by_f64 in [(0, False), (4, False), (5, True)]:
        for desc in (True, False):
            for limit in (1, 3, 6, 50):
                check(t.aggregate_topn(tpl.aggs, tpl.group_by, tpl.where, agg, desc, limit),
                      expected(full, agg, desc, limit, by_f64))
    s = workloads.selective_scan_sum()
    g = t.aggregate_topn(s.aggs, (), s.where, 0, True, 5)
    same_query(g, oracle.aggregate(host, CT, s.aggs, (), s.where))
    t.drop()


def test_topn_of_the_join(ctx):
    dim = datagen.dimension(30_000, seed=21)
    fact = datagen.fact_fk(200_000, 30_000, 0.8, seed=22)
    fct = {**datagen.LINEITEM_COLTYPES, "fk": "int"}
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    f = ctx.register(fact, fct)
    tpl = workloads.join_group_agg()
    j = d.join_build("key", tpl.build_where)
    full = oracle.aggregate(fact, fct, tpl.aggs, tpl.group_by, None,
                            build=(dim, datagen.DIMENSION_COLTYPES, "key", tpl.build_where), probe_key="fk")
    check(f.aggregate_topn(tpl.aggs, tpl.group_by, None, 0, True, 5, join=j, probe_key="fk"),
          expected(full, 0, True, 5, False))
    j.drop()
