"""The join's build side is chosen the reference's way (the side with fewer
rows after its own filter, hash_join_with_keys join.rs:557-575): with a
selective fact filter the fact side is built (duplicate keys: the hash-probe
path), with the usual filters the dimension is; either way the aggregate and
the (fact row, dimension row) pairs equal the oracle's."""
import numpy as np
import pytest

import oracle
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import build_col, col, count_star, sum_

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES
FCT = {**CT, "fk": "int"}


def same_query(a, b):
    assert a.rows_selected == b.rows_selected and a.keys == b.keys
    for ra, rb in zip(a.values, b.values):
        assert [(x.value, x.count) for x in ra] == [(y.value, y.count) for y in rb]


@pytest.mark.parametrize("fact_where, built", [(None, "b"), (col("quantity") < 2, "a"),
                                               (col("ship_day") < datagen.DAY0 + 30, "a")])
def test_build_side_follows_filtered_sizes(ctx, fact_where, built):
    fact = datagen.fact_fk(400_000, 40_000, 0.8, seed=81)
    dim = datagen.dimension(40_000, seed=82)
    f = ctx.register(fact, FCT)
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    tj = workloads.join_group_agg()
    plan = ctx.join_smaller(f, "fk", fact_where, d, "key", tj.build_where)
    assert plan.build_is_a == (built == "a")
    assert plan.rows_a == oracle.filter(fact, FCT, fact_where).count
    assert plan.rows_b == oracle.filter(dim, datagen.DIMENSION_COLTYPES, tj.build_where).count
    build = (dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
    for aggs, gb in ((tj.aggs, tj.group_by),
                     ([count_star(), sum_(col("quantity") * build_col("order_day"))], (build_col("segment"), "flag_a"))):
        got = plan.aggregate(aggs, gb, group_cap=1 << 12)
        exp = oracle.aggregate(fact, FCT, aggs, gb, fact_where, build=build, probe_key="fk")
        # rows_selected is the probe side's filtered count: compare the groups.
        assert got.keys == exp.keys
        for ra, rb in zip(got.values, exp.values):
            assert [(x.value, x.count) for x in ra] == [(y.value, y.count) for y in rb]
    fr, dr = plan.pairs()
    ofr, odr = oracle.join_pairs(fact, FCT, "fk", fact_where, dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)
    order, oorder = np.lexsort((dr, fr)), np.lexsort((odr, ofr))
    assert np.array_equal(fr[order], ofr[oorder]) and np.array_equal(dr[order], odr[oorder])
    plan.drop()
    f.drop()
    d.drop()
