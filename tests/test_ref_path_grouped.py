"""The restated reference CPU paths of the grouped and high-cardinality
queries (oracle/ref_path.cpp) against the exact oracle and the f64
emulation: integer sums and counts exact, f64 sums bit-identical to the
reference's arithmetic in row order."""
import numpy as np

import oracle
from oracle import f64_emulation as F
from oracle import refpath
from turbogp_b200 import datagen, workloads

CT = datagen.LINEITEM_COLTYPES


def test_grouped_q1_matches_exact_and_f64_emulation():
    n = 700_003
    host = datagen.lineitem(n, seed=3)
    tpl = workloads.filtered_group_agg()
    for threads in (1, 4):
        r = refpath.grouped_q1(host, tpl, CT, threads=threads)
        exact = oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where)
        sel = oracle.filter(host, CT, tpl.where).rowids.astype(np.int64)
        c, k, mul, sub, add = F.c, F.k, F.mul, F.sub, F.add
        dp = mul(c("price_cents"), sub(k(100), c("discount_pct")))
        keys, counts, sums, avgs = F.grouped(host, sel, tpl.group_by, [dp, mul(dp, add(k(100), c("tax_pct")))],
                                             [c("quantity")])
        assert [g[0] for g in r["groups"]] == list(exact.keys) == keys
        for g, vals, i in zip(r["groups"], exact.values, range(len(keys))):
            _, cnt, sq, sp, fdp, fch, aq = g
            assert cnt == vals[0].value == counts[i]
            assert sq == vals[1].value and sp == vals[2].value
            assert fdp == sums[0][i] and fch == sums[1][i] and aq == avgs[0][i]


def test_highcard_matches_exact():
    n = 400_000
    h = datagen.highcard(n, 200_000, 1.1, seed=9)
    for threads in (1, 3):
        r = refpath.highcard(h, threads=threads)
        exact = oracle.aggregate(h, None, workloads.highcard_group().aggs, ("key",))
        assert r["ngroups"] == len(exact.keys)
        assert [int(x) for x in r["keys"]] == [k[0] for k in exact.keys]
        assert [int(x) for x in r["counts"]] == [v[0].value for v in exact.values]
        assert [int(x) for x in r["sums"]] == [v[1].value for v in exact.values]


def test_join_group_matches_exact():
    dim = datagen.dimension(60_000, seed=12)
    fact = datagen.fact_fk(500_000, 60_000, 0.8, seed=13)
    fact["fk"][:40] = 90_000   # keys outside the build side
    tpl = workloads.join_group_agg(order_day_lt=datagen.DAY0 + datagen.NDAYS // 2)
    fct = {"fk": "int", "price_cents": "int", "discount_pct": "int"}
    exact = oracle.aggregate({k: fact[k] for k in fct}, fct, tpl.aggs, tpl.group_by, None,
                             build=(dim, datagen.DIMENSION_COLTYPES, "key", tpl.build_where), probe_key="fk")
    for threads in (1, 4):
        r = refpath.join_group(fact, dim, datagen.DAY0 + datagen.NDAYS // 2, threads=threads)
        assert [g[0] for g in r["groups"]] == [k[0] for k in exact.keys]
        for (seg, cnt, s), vals in zip(r["groups"], exact.values):
            assert cnt == vals[1].value
            assert vals[0].value < 2**53 and s == float(vals[0].value)   # exact below 2^53
