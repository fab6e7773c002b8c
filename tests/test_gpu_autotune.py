"""The autotuner (tgp_autotune) on the GPU: every candidate variant of a
query class (threads x stage cap x accumulator placement / dense programs, or
x pre-aggregation for hash grouping) returns the planner's result bit for
bit and the oracle's; the fastest is installed for the class, later queries
of the class run it and still match the oracle, and the tuned entries survive
a save / load round trip."""
import pytest

import oracle
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import Context, col, count_star, sum_

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES


def same_query(a, b):
    assert a.rows_selected == b.rows_selected and a.keys == b.keys
    for ra, rb in zip(a.values, b.values):
        for x, y in zip(ra, rb):
            assert (x.value, x.count) == (y.value, y.count)
            assert x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)


def check_report(rep, min_candidates):
    cands = rep["candidates"]
    assert len(cands) >= min_candidates
    ran = [c for c in cands if c["status"] == 0]
    assert ran and all(c["same_result"] for c in ran)
    assert rep["best_ms"] == min(c["ms"] for c in ran)


def test_autotune_grouped_scalar_join_and_hash(tmp_path):
    host = datagen.lineitem(700_001, seed=41)
    dim = datagen.dimension(20_000, seed=42)
    fact = datagen.fact_fk(500_000, 20_000, 0.8, seed=43)
    hc = datagen.highcard(600_000, 100_000, 1.1, seed=44)
    fct = {**CT, "fk": "int"}
    with Context(0) as ctx:
        t = ctx.register(host, CT)
        d, f, h = ctx.register(dim, datagen.DIMENSION_COLTYPES), ctx.register(fact, fct), ctx.register(hc)
        tj = workloads.join_group_agg()
        j = d.join_build("key", tj.build_where)
        cases = []
        for tpl in (workloads.filtered_group_agg(), workloads.selective_scan_sum()):
            cases.append((t.prepare(tpl.aggs, tpl.group_by, tpl.where),
                          lambda tpl=tpl: oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where), 10))
        cases.append((f.prepare(tj.aggs, tj.group_by, None, join=j, probe_key="fk"),
                      lambda: oracle.aggregate(fact, fct, tj.aggs, tj.group_by, None,
                                               build=(dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where),
                                               probe_key="fk"), 10))
        aggs = [count_star(), sum_(col("value"))]
        cases.append((h.prepare(aggs, ("key",), col("value") < 900, group_cap=1 << 20),
                      lambda: oracle.aggregate(hc, None, aggs, ("key",), col("value") < 900), 6))
        for pq, expect, mincand in cases:
            rep = ctx.autotune(pq, reps=3)
            check_report(rep, mincand)
            assert rep["class"] in ctx.tuned_variants()
            same_query(pq.run(), expect())
        saved = ctx.tuned_variants()
        path = tmp_path / "tuning.json"
        ctx.save_tuning(path)
        j.drop()
    with Context(0) as ctx2:
        assert ctx2.load_tuning(path) == len(saved)
        assert ctx2.tuned_variants() == saved
        t2 = ctx2.register(host, CT)
        tpl = workloads.filtered_group_agg()
        same_query(t2.aggregate(tpl.aggs, tpl.group_by, tpl.where),
                   oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where))


def test_default_variant_knobs_give_the_same_results():
    host = datagen.lineitem(300_007, seed=45)
    tpl = workloads.filtered_group_agg()
    expect = oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where)
    with Context(0) as ctx:
        t = ctx.register(host, CT)
        for knobs in ({"threads": 256, "max_stages": 2}, {"placement": 2}, {"placement": 3},
                      {"placement": 1, "dense": 0}, {"shapes": 0}, {"ctas_per_sm": 2, "max_stages": 2}):
            ctx.set_default_variant(**knobs)
            same_query(t.aggregate(tpl.aggs, tpl.group_by, tpl.where), expect)
            ctx.set_default_variant(threads=0, max_stages=8, placement=0, presum=1, dense=1, shapes=1, payload=1,
                                    ctas_per_sm=1, l2_ahead=0)
