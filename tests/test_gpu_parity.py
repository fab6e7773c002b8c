"""GPU results against the CPU oracle on seeded inputs: bit-exact bitmaps,
row ids, join pairs, counts and int128 sums."""
import numpy as np
import pytest

import oracle
from turbogp_b200 import _capi as A
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import avg, build_col, col, count_col, count_star, max_, min_, sum_

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 7, 31, 32, 33, 255, 2047, 2048, 2049, 4096, 10_007, 100_003]
CT = datagen.LINEITEM_COLTYPES


def bits(bm, n):
    return np.unpackbits(bm, bitorder="little")[:n]


def same_query(a, b):
    assert a.rows_selected == b.rows_selected
    assert a.keys == b.keys
    assert len(a.values) == len(b.values)
    for ga, gb in zip(a.values, b.values):
        for x, y in zip(ga, gb):
            assert x.count == y.count
            if x.count:
                assert x.value == y.value
                assert x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)


def predicates(d0=datagen.DAY0):
    c = col
    return [
        None,
        c("ship_day") <= d0 + 2435,
        (c("ship_day") >= d0 + 730) & (c("ship_day") < d0 + 1095) & c("discount_pct").between(5, 7) & (c("quantity") < 24),
        (c("flag_a") == 1) | (c("flag_b") == 0),
        ~((c("quantity") > 10) & (c("price_cents") <= 5_000_000)) | c("tax_pct").not_between(2, 6),
        c("price_cents") != 1_000_000,
        (c("quantity") < -5) | (c("discount_pct") >= 11),        # nothing passes
        c("quantity") >= -(2**40),                                # everything passes (literal beyond i32)
        c("ship_day") < 2**40,                                    # DATE compare, literal beyond i32
        (c("flag_a") <= 300) & (c("flag_b") >= -1),
    ]


@pytest.mark.parametrize("n", SIZES)
def test_filter_bitmaps_and_rowids(ctx, n):
    t_host = datagen.lineitem(n, seed=11 + n)
    t = ctx.register(t_host, CT)
    for i, p in enumerate(predicates()):
        g = t.filter(p)
        o = oracle.filter(t_host, CT, p)
        assert g.count == o.count, (n, i)
        assert np.array_equal(bits(g.bitmap, n), bits(o.bitmap, n)), (n, i)
        if n:
            # tail bits beyond n are zero
            assert np.all(np.unpackbits(g.bitmap, bitorder="little")[n:] == 0)
        assert np.array_equal(g.rowids, o.rowids), (n, i)
    t.drop()


def test_filter_all_dtypes_and_signedness(ctx):
    rng = np.random.default_rng(5)
    n = 5000
    cols = {
        "u8": rng.integers(0, 256, n, dtype=np.uint8),
        "i32": rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32),
        "i64": rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64),
        "u64": rng.integers(0, 2**64 - 1, n, dtype=np.uint64),
        "f64": rng.normal(0, 100, n),
    }
    cols["i32"][:4] = [-2**31, 2**31 - 1, 0, -1]
    cols["i64"][:4] = [-2**63, 2**63 - 1, 0, -1]
    for ct_name in ["int", "date"]:
        cts = {k: ct_name for k in ["u8", "i32", "i64", "u64"]}
        cts["f64"] = "float"
        t = ctx.register(cols, cts)
        for name in ["u8", "i32", "i64", "u64"]:
            for v in [0, 1, -1, 7, 200, 255, 256, -2**31, 2**31 - 1, 2**31, -2**63, 2**63 - 1, 2**64 - 1]:
                for op in ["__eq__", "__ne__", "__lt__", "__le__", "__gt__", "__ge__"]:
                    p = getattr(col(name), op)(v)
                    assert t.filter(p, rowids=False).count == oracle.filter(cols, cts, p).count, (ct_name, name, v, op)
                for lo, hi in [(-5, 5), (10, 3), (0, 2**64 - 1), (-2**63, 2**63 - 1)]:
                    for p in [col(name).between(lo, hi), col(name).not_between(lo, hi)]:
                        g = t.filter(p)
                        o = oracle.filter(cols, cts, p)
                        assert np.array_equal(g.rowids, o.rowids), (ct_name, name, lo, hi)
        for v in [0.0, 1.5, -3.25, 100.0]:
            for op in ["__eq__", "__ne__", "__lt__", "__le__", "__gt__", "__ge__"]:
                p = getattr(col("f64"), op)(v)
                assert np.array_equal(t.filter(p).rowids, oracle.filter(cols, cts, p).rowids), (v, op)
        t.drop()


@pytest.mark.parametrize("n", [0, 1, 2049, 100_003, 1_000_000])
def test_templates_match_oracle(ctx, n):
    t_host = datagen.lineitem(n, seed=3)
    t = ctx.register(t_host, CT)
    for tpl in [workloads.filtered_group_agg(), workloads.selective_scan_sum()]:
        g = t.aggregate(tpl.aggs, tpl.group_by, tpl.where)
        o = oracle.aggregate(t_host, CT, tpl.aggs, tpl.group_by, tpl.where)
        same_query(g, o)
    t.drop()


def test_group_modes(ctx):
    """Direct private / shared / global tables and the global hash table."""
    n = 300_000
    t_host = datagen.lineitem(n, seed=21)
    t = ctx.register(t_host, CT)
    aggs = [count_star(), sum_(col("price_cents") * (100 - col("discount_pct"))), min_(col("quantity")),
            max_(col("price_cents")), avg(col("quantity")), count_col(col("discount_pct"))]
    for gb in [("flag_a",), ("flag_a", "flag_b"), ("tax_pct", "flag_a", "flag_b"), ("ship_day",),
               ("ship_day", "quantity"), ("price_cents",), ("quantity", "price_cents")]:
        g = t.aggregate(aggs, gb, col("discount_pct") <= 8)
        o = oracle.aggregate(t_host, CT, aggs, gb, col("discount_pct") <= 8)
        same_query(g, o)
    t.drop()


def test_int128_sums_and_overflow_flag(ctx):
    n = 100_000
    big = np.full(n, 2**62 + 12345, dtype=np.int64)
    grp = (np.arange(n) % 3).astype(np.uint8)
    cols = {"v": big, "g": grp, "neg": -big}
    t = ctx.register(cols)
    for aggs in [[sum_(col("v")), sum_(col("neg")), count_star()], [sum_(col("v") * 3)], [sum_(col("v") * col("v"))]]:
        for gb in [(), ("g",)]:
            g = t.aggregate(aggs, gb)
            o = oracle.aggregate(cols, None, aggs, gb)
            same_query(g, o)
            assert g.flags == o.flags
    t.drop()


def test_join_pairs_and_join_aggregate(ctx):
    dim = datagen.dimension(50_000, seed=7)
    fact = datagen.fact_fk(400_000, 50_000, 0.8, seed=8)
    fact["fk"][:100] = 60_000  # keys beyond the build side
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    f = ctx.register(fact, {**CT, "fk": "int"})
    tpl = workloads.join_group_agg()
    j = d.join_build("key", tpl.build_where)
    pr, br = j.probe_pairs(f, "fk", col("quantity") < 30)
    opr, obr = oracle.join_pairs(fact, {**CT, "fk": "int"}, "fk", col("quantity") < 30, dim,
                                 datagen.DIMENSION_COLTYPES, "key", tpl.build_where)
    assert np.array_equal(pr, opr) and np.array_equal(br, obr)
    for where in [None, col("quantity") < 30]:
        g = f.aggregate(tpl.aggs, tpl.group_by, where, join=j, probe_key="fk")
        o = oracle.aggregate(fact, {**CT, "fk": "int"}, tpl.aggs, tpl.group_by, where,
                             build=(dim, datagen.DIMENSION_COLTYPES, "key", tpl.build_where), probe_key="fk")
        same_query(g, o)
    # Scalar aggregate over the join and duplicate build keys.
    dup = {"key": np.repeat(np.arange(1, 1001, dtype=np.int32), 3), "w": np.arange(3000, dtype=np.int32)}
    dd = ctx.register(dup)
    jd = dd.join_build("key")
    aggs = [count_star(), sum_(col("price_cents") * build_col("w"))]
    small = {k: v[:20_000] for k, v in fact.items()}
    fs = ctx.register(small, {**CT, "fk": "int"})
    g = fs.aggregate(aggs, (), None, join=jd, probe_key="fk")
    o = oracle.aggregate(small, {**CT, "fk": "int"}, aggs, (), None, build=(dup, None, "key", None), probe_key="fk")
    same_query(g, o)
    pr, br = jd.probe_pairs(fs, "fk")
    opr, obr = oracle.join_pairs(small, {**CT, "fk": "int"}, "fk", None, dup, None, "key", None)
    assert np.array_equal(pr, opr) and np.array_equal(br, obr)


def test_full_size_selective_scan(ctx):
    """The 60M-row scan workload at full size against the oracle."""
    n = 60_000_000
    t_host = datagen.lineitem(n, seed=1)
    t = ctx.register(t_host, CT)
    tpl = workloads.selective_scan_sum()
    g = t.aggregate(tpl.aggs, tpl.group_by, tpl.where)
    o = oracle.aggregate(t_host, CT, tpl.aggs, tpl.group_by, tpl.where)
    same_query(g, o)
    # Size-independent property: the filter's count equals the aggregate's count.
    assert t.filter(tpl.where, bitmap=False, rowids=False).count == g.values[0][1].value
    t.drop()


def test_dense_value_programs(ctx):
    """Grouped aggregates whose value lists share factor prefixes, constants,
    MIN / MAX / COUNT(col), 0-2 group keys, at selectivities that mix dense and
    sparse warps, with tails, against the oracle."""
    from turbogp_b200.engine import lit
    p, d, t, q = col("price_cents"), col("discount_pct"), col("tax_pct"), col("quantity")
    programs = [
        [count_star(), sum_(q), sum_(p), sum_(p * (100 - d)), sum_(p * (100 - d) * (100 + t)), avg(q)],
        [sum_(p * d), sum_(p * d * 3), min_(p * d), max_(q - 60), count_col(d - 5)],
        [sum_(lit(7)), sum_(q * (-3)), sum_(-q + 11), sum_(q * q * q), max_(d), sum_(p)],
        [min_(q), max_(q), sum_(q), count_star()],
        [sum_(p * t * d * q)],
    ]
    keys = [(), ("flag_a",), ("flag_a", "flag_b"), ("tax_pct", "flag_b"), ("discount_pct",)]
    wheres = [None, col("ship_day") <= datagen.DAY0 + 1500, col("quantity") <= 15, col("discount_pct") == 3]
    for n in [2048 * 37 + 5, 250_000]:
        t_host = datagen.lineitem(n, seed=31 + n)
        t_host["price_cents"][::7] *= -1          # negative values and products
        tb = ctx.register(t_host, CT)
        for aggs in programs:
            for gb in keys:
                for w in wheres:
                    g = tb.aggregate(aggs, gb, w)
                    o = oracle.aggregate(t_host, CT, aggs, gb, w)
                    same_query(g, o)
        tb.drop()


def test_dense_flushes_near_int64_bound(ctx):
    """Per-row values near 2^60 force the int64 partials to flush every few
    rows; sums stay exact in int128."""
    n = 400_003
    rng = np.random.default_rng(5)
    cols = {"v": rng.integers(2**59, 2**60, n, dtype=np.int64),
            "w": rng.integers(-2**60, -2**59, n, dtype=np.int64),
            "g": rng.integers(0, 5, n, dtype=np.uint8),
            "s": rng.integers(0, 100, n, dtype=np.int32)}
    tb = ctx.register(cols)
    aggs = [count_star(), sum_(col("v")), sum_(col("w")), max_(col("v"))]
    for gb in [(), ("g",)]:
        for w in [None, col("s") < 70]:
            g = tb.aggregate(aggs, gb, w)
            o = oracle.aggregate(cols, None, aggs, gb, w)
            same_query(g, o)
    tb.drop()


def test_join_payload_and_hash_probe_paths(ctx):
    """Joined aggregates through the unique-key payload array (dense build key
    range) and through the hash table (duplicate keys, sparse key range), with
    build-side, probe-side and mixed group keys."""
    nb, n = 40_000, 300_000
    dim = datagen.dimension(nb, seed=17)
    fact = datagen.fact_fk(n, nb, 0.8, seed=18)
    fact["fk"][::97] = nb + 5          # keys past the build range
    fact["fk"][::89] = 0               # keys below it
    fct = {**CT, "fk": "int"}
    f = ctx.register(fact, fct)
    variants = {
        "dense": dim,
        "sparse": {**dim, "key": (dim["key"].astype(np.int64) * 1_000_003).astype(np.int64)},
        "dup": {**dim, "key": (dim["key"] // 2 + 1).astype(np.int32)},
    }
    p, d = col("price_cents"), col("discount_pct")
    agg_sets = [[sum_(p * (100 - d)), count_star(), max_(col("quantity")), sum_(col("quantity"))],
                [sum_(p * (100 - d)), count_star()]]          # the join template's own shape
    for name, dh in variants.items():
        probe = dict(fact)
        if name == "sparse":
            probe = {**fact, "fk": (fact["fk"].astype(np.int64) * 1_000_003)}
        fp = ctx.register(probe, fct) if name == "sparse" else f
        dt = ctx.register(dh, datagen.DIMENSION_COLTYPES)
        j = dt.join_build("key", col("order_day") < datagen.DAY0 + datagen.NDAYS // 2)
        for gb, aggs in [(g, a) for g in [(build_col("segment"),), (), (build_col("segment"), "flag_a"), ("flag_b",)]
                         for a in agg_sets]:
            for where in [None, col("quantity") < 30]:
                g = fp.aggregate(aggs, gb, where, join=j, probe_key="fk")
                o = oracle.aggregate(probe, fct, aggs, gb, where,
                                     build=(dh, datagen.DIMENSION_COLTYPES, "key",
                                            col("order_day") < datagen.DAY0 + datagen.NDAYS // 2),
                                     probe_key="fk")
                same_query(g, o)
        j.drop()
        dt.drop()
        if fp is not f:
            fp.drop()
    f.drop()


def test_hash_grouping_hot_keys_and_device_format(ctx):
    """Zipf keys through direct global grouping and hash grouping (shared
    pre-aggregation of hot keys in both, then the global tables), multi-key
    tuples, hash results sorted and formatted on the device; large values
    switch the pre-aggregation off."""
    n = 2_000_003
    h = datagen.highcard(n, 200_000, 1.1, seed=9)
    rng = np.random.default_rng(3)
    h["k2"] = rng.integers(-3, 4, n, dtype=np.int32)
    h["big"] = rng.integers(-2**40, 2**40, n, dtype=np.int64)
    h["wide"] = h["key"] * 50          # a key range past the direct-indexed limit: hash grouping
    t = ctx.register(h)
    cases = [
        ([count_star(), sum_(col("value")), count_col(col("value"))], ("wide",), None),
        ([count_star(), sum_(col("big"))], ("wide",), col("value") < 700),
        ([count_star(), sum_(col("value")), avg(col("value")), count_col(col("value"))], ("key",), None),
        ([count_star(), sum_((col("value") - 7) * 3)], ("key", "k2"), col("value") < 900),
        ([sum_(col("big")), count_star(), min_(col("value"))], ("key",), None),
        ([count_star()], ("k2", "key"), col("value") >= 500),
    ]
    for aggs, gb, where in cases:
        g = t.aggregate(aggs, gb, where, group_cap=1 << 20)
        o = oracle.aggregate(h, None, aggs, gb, where)
        same_query(g, o)
    t.drop()


def test_one_word_direct_slots(ctx):
    """GROUP BY one key over a moderate range with COUNT(*) and one SUM or
    COUNT(col): the count and the biased sum share one 64-bit word per key
    when the host proves they never meet. Negative keys and values (a
    negative bias), an affine argument, count only, COUNT(col), the shared
    pre-aggregation switched off by large values, a partial last tile, and
    a value range too wide to share a word (the four-word slots again)."""
    # Keys spread over a range past the direct-indexed accumulators' limit
    # (2^22 groups) and below twice the rows: a slot per key value.
    n = 2_500_003
    h = datagen.highcard(n, 200_000, 1.1, seed=11)
    h["key"] = h["key"] * 23
    rng = np.random.default_rng(5)
    h["negkey"] = h["key"] - 2_300_000
    h["big"] = rng.integers(-2**40, 2**40, n, dtype=np.int64)
    assert 1 << 22 < int(h["key"].max() - h["key"].min()) + 1 <= 2 * n
    t = ctx.register(h)
    v = col("value")
    cases = [
        ([count_star(), sum_(v)], ("key",), None),
        ([count_star(), sum_(v - 500), avg(v - 500)], ("negkey",), v < 900),
        ([count_star()], ("key",), None),
        ([count_col(v), count_star()], ("negkey",), v >= 3),
        ([count_star(), sum_(v * 300)], ("key",), None),           # one word, no shared pre-aggregation
        ([count_star(), sum_(v * 3000)], ("key",), None),          # too wide for one word at 2.5M rows
        ([sum_(col("big")), count_star()], ("key",), None),         # range too wide for one word
    ]
    for aggs, gb, where in cases:
        g = t.aggregate(aggs, gb, where, group_cap=1 << 20)
        o = oracle.aggregate(h, None, aggs, gb, where)
        same_query(g, o)
    t.drop()


def test_batch_persistent_launch_matches_single_queries(ctx):
    """A batch of queries of uneven sizes and all three templates (scan +
    scalar sum, grouped Q1 shape, join + group) through the persistent
    launch, plus hash-grouped and empty queries that run alone: each result
    equals the oracle's, whatever morsels the CTAs took."""
    rng = np.random.default_rng(12)
    sizes = [0, 1, 2047, 2049, 70_001, 1_000_003, 3_000_000]
    tabs = {n: datagen.lineitem(n, seed=100 + i) for i, n in enumerate(sizes)}
    regs = {n: ctx.register(h, CT) for n, h in tabs.items()}
    dim = datagen.dimension(30_000, seed=5)
    fact = datagen.fact_fk(500_000, 30_000, 0.8, seed=6)
    fct = {**CT, "fk": "int"}
    d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    f = ctx.register(fact, fct)
    tj = workloads.join_group_agg()
    j = d.join_build("key", tj.build_where)
    pqs, expect = [], []
    for k in range(40):
        n = sizes[k % len(sizes)]
        kind = k % 4
        if kind == 0:
            tpl = workloads.selective_scan_sum(day_lo=datagen.DAY0 + int(rng.integers(0, 2000)),
                                               days=int(rng.integers(1, 500)), qty_lt=int(rng.integers(1, 51)))
        elif kind == 1:
            tpl = workloads.filtered_group_agg(ship_max=datagen.DAY0 + int(rng.integers(0, datagen.NDAYS)))
        elif kind == 2:
            tpl = None
        else:
            tpl = workloads.filtered_group_agg()
            tpl.group_by = ("price_cents",)                       # hash grouping: runs alone
        if tpl is None:
            where = col("quantity") < int(rng.integers(1, 51))
            pqs.append(f.prepare(tj.aggs, tj.group_by, where, join=j, probe_key="fk"))
            expect.append(oracle.aggregate(fact, fct, tj.aggs, tj.group_by, where,
                                           build=(dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where),
                                           probe_key="fk"))
            continue
        pqs.append(regs[n].prepare(tpl.aggs, tpl.group_by, tpl.where, group_cap=1 << 20))
        expect.append(oracle.aggregate(tabs[n], CT, tpl.aggs, tpl.group_by, tpl.where))
    outs = ctx.submit(pqs).wait()
    assert len(outs) == len(pqs)
    for o, e in zip(outs, expect):
        same_query(o, e)
    # Polling form, and the same queries again (plans and buffers reused).
    h = ctx.submit(pqs[:9])
    while not h.poll():
        pass
    for o, e in zip(h.wait(), expect[:9]):
        same_query(o, e)
    j.drop()


def test_join_payload_widths_and_shapes(ctx):
    """Payload joins with no probe-side predicate, grouped by build-side keys:
    25 groups (u8 payload entries), 2,526 and 25 x 2,526 groups (u16, then
    u32 entries), one- and two-factor sums, two values, count only, keys
    outside the build range, and a partial last tile."""
    nb, n = 30_000, 1_000_037
    dim = datagen.dimension(nb, seed=27)
    fact = datagen.fact_fk(n, nb, 0.8, seed=28)
    fact["fk"][::101] = nb + 9
    fact["fk"][::103] = -4
    fct = {**CT, "fk": "int"}
    f = ctx.register(fact, fct)
    dt = ctx.register(dim, datagen.DIMENSION_COLTYPES)
    bw = col("order_day") < datagen.DAY0 + datagen.NDAYS // 3
    j = dt.join_build("key", bw)
    p, d, q = col("price_cents"), col("discount_pct"), col("quantity")
    cases = [
        ((build_col("segment"),), [sum_(p * (100 - d)), count_star()]),
        ((build_col("segment"),), [count_star()]),
        ((build_col("order_day"),), [sum_(q), count_star(), sum_((p - 7) * (d + 3))]),
        ((build_col("segment"), build_col("order_day")), [sum_(p), count_star()]),
        ((), [sum_(p * d), count_star(), avg(q)]),
    ]
    for gb, aggs in cases:
        g = f.aggregate(aggs, gb, None, join=j, probe_key="fk")
        o = oracle.aggregate(fact, fct, aggs, gb, None, build=(dim, datagen.DIMENSION_COLTYPES, "key", bw),
                             probe_key="fk")
        same_query(g, o)
    j.drop()
    dt.drop()
    f.drop()


@pytest.mark.parametrize("n", [0, 5, 127, 128, 1_000_003])
def test_q1_shape_streaming_predicates(ctx, n):
    """The TPC-H Q1 shape (GROUP BY two u8 flags, count and four sums) under
    no predicate, one to four int32 leaves, a negated leaf, and a leaf kind
    the streaming kernel does not take (u8 column: the scan kernel runs),
    with row counts below, at and past a 128-row chunk."""
    h = datagen.lineitem(n, seed=41 + n)
    t = ctx.register(h, CT)
    tpl = workloads.filtered_group_agg()
    d0, c = datagen.DAY0, col
    wheres = [None,
              c("ship_day") <= d0 + 2000,
              (c("ship_day") >= d0 + 300) & (c("ship_day") < d0 + 2100) & c("discount_pct").between(2, 8) &
              (c("quantity") < 40) & (c("tax_pct") > 1),
              ~(c("tax_pct") < 3) & (c("quantity") > 5),
              (c("flag_a") == 1) & (c("ship_day") <= d0 + 2400)]
    for w in wheres:
        g = t.aggregate(tpl.aggs, tpl.group_by, w)
        o = oracle.aggregate(h, CT, tpl.aggs, tpl.group_by, w)
        same_query(g, o)
    t.drop()


def test_footprint_counts_one_word_slots(ctx):
    """The admission estimate (tgp_query_footprint) sizes the group table the
    way the run lays it out: one word per key value when COUNT(*) and the SUM
    share a word, four when the value range is too wide for that; the rest of
    the estimate (result block, format scratch, formatted groups) is the
    same for both."""
    n = 2_500_003
    h = datagen.highcard(n, 200_000, 1.1, seed=13)
    h["key"] = h["key"] * 23   # a key range past 2^22 groups: one slot per key value
    h["big"] = np.random.default_rng(2).integers(-2**40, 2**40, n, dtype=np.int64)
    t = ctx.register(h)
    packed = t.prepare([count_star(), sum_(col("value"))], ("key",), None, group_cap=1 << 18).footprint()
    wide = t.prepare([count_star(), sum_(col("big"))], ("key",), None, group_cap=1 << 18).footprint()
    keys = int(h["key"].max() - h["key"].min() + 1)
    assert 1 << 22 < keys <= 2 * n
    assert wide - packed == max(16, keys) * 3 * 8
    t.drop()
