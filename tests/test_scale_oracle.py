"""The at-scale numpy checker (oracle/scale.py) agrees with the row-at-a-time
oracle on every benchmark template, on predicates of every comparison kind,
on the join and on high-cardinality grouping — so the full-size GPU tests
that use it are checked against the same semantics."""
import numpy as np
import pytest

import oracle
from oracle import scale
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import avg, build_col, col, count_col, count_star, max_, min_, sum_

CT = datagen.LINEITEM_COLTYPES


def same(a, b):
    assert a.rows_selected == b.rows_selected
    assert a.keys == b.keys
    for ra, rb in zip(a.values, b.values):
        for x, y in zip(ra, rb):
            assert (x.value, x.count) == (y.value, y.count)
            assert x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)


@pytest.mark.parametrize("n", [0, 1, 33, 2049, 50_003])
def test_templates_match_the_oracle(n):
    host = datagen.lineitem(n, seed=5 + n)
    for tpl in (workloads.filtered_group_agg(), workloads.selective_scan_sum(),
                workloads.selective_scan_sum(day_lo=datagen.DAY0 + 17, days=40, disc_lo=0, disc_hi=3, qty_lt=7)):
        same(scale.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where),
             oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where))


def test_predicates_and_aggregate_kinds_match_the_oracle():
    host = datagen.lineitem(20_011, seed=9)
    c = col
    wheres = [
        None,
        (c("flag_a") == 1) | (c("flag_b") != 0),
        ~((c("quantity") > 10) & (c("price_cents") <= 5_000_000)) | c("tax_pct").not_between(2, 6),
        c("quantity") >= -(2 ** 40),
        c("ship_day") < 2 ** 40,
        (c("quantity") < -5) | (c("discount_pct") >= 11),
    ]
    aggs = [count_star(), sum_(c("quantity") * (c("price_cents") - 7)), min_(c("discount_pct") - 3),
            max_(-c("price_cents")), count_col(c("discount_pct")), avg((c("tax_pct") + 1) * 3)]
    for w in wheres:
        for gb in ((), ("flag_a",), ("flag_b", "tax_pct"), ("ship_day",)):
            same(scale.aggregate(host, CT, aggs, gb, w), oracle.aggregate(host, CT, aggs, gb, w))


def test_join_matches_the_oracle():
    nb, n = 4_000, 30_011
    dim = datagen.dimension(nb, seed=21)
    fact = datagen.fact_fk(n, nb + 300, 0.8, seed=22)  # some foreign keys have no build row
    fct = {**CT, "fk": "int"}
    tj = workloads.join_group_agg(order_day_lt=datagen.DAY0 + 900)
    for gb, aggs in ((tj.group_by, tj.aggs),
                     ((build_col("segment"), "flag_a"), [count_star(), sum_(build_col("order_day") * col("quantity"))])):
        build = (dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
        same(scale.aggregate(fact, fct, aggs, gb, col("quantity") < 30, build=build, probe_key="fk"),
             oracle.aggregate(fact, fct, aggs, gb, col("quantity") < 30, build=build, probe_key="fk"))


def test_high_cardinality_grouping_matches_the_oracle():
    host = datagen.highcard(200_003, 50_000, 1.1, seed=31)
    o = oracle.aggregate(host, None, [count_star(), sum_(col("value"))], ("key",))
    k, cnt, s = scale.group_count_sum(host["key"], host["value"])
    assert k.tolist() == [kk[0] for kk in o.keys]
    assert cnt.tolist() == [r[0].value for r in o.values]
    assert s.tolist() == [r[1].value for r in o.values]
    same(scale.aggregate(host, None, [count_star(), sum_(col("value"))], ("key",)), o)
