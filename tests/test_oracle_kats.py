"""The CPU oracle against the known answers of the reference's own tests."""
import numpy as np
import pytest

import oracle
from kat_helpers import arith_aggs, kernel_params, leaf, scalar_expect
from conftest import gen_column
from turbogp_b200 import _capi as A
from turbogp_b200.engine import col, count_star, sum_, avg
from turbogp_b200.kernel_table import Operator


def test_filter_kats(kats):
    for c in kats["filters"]:
        x = gen_column(c["column"], c["dtype"])
        out = oracle.filter({"c": x}, {"c": c["coltype"]}, leaf("c", c["cmp"], c["lit"]))
        if c["expect"] == "scalar":
            exp = scalar_expect(x, c["cmp"], c["lit"])
            assert out.count == int(exp.sum()), c["source"]
            assert np.array_equal(np.unpackbits(out.bitmap, bitorder="little")[: len(x)].astype(bool), exp)
        elif isinstance(c["expect"], list):
            bits = np.unpackbits(out.bitmap, bitorder="little")[: len(x)].astype(bool).tolist()
            assert bits == c["expect"], c["source"]
        else:
            assert out.count == c["expect"], c["source"]


def test_conjunction_kats(kats):
    for c in kats["conjunctions"]:
        x = gen_column(c["column"], c["dtype"])
        (o1, v1), (o2, v2) = c["leaves"]
        out = oracle.filter({"c": x}, {"c": c["coltype"]}, leaf("c", o1, v1) & leaf("c", o2, v2))
        assert out.count == c["count"], c["source"]


def test_scan_kernel_kats(kats):
    for c in kats["scan_kernels"]:
        cells = gen_column(c["cells"], "u64")
        n, _, mask = oracle.kernel_execute(int(Operator[c["op"]]), cells, kernel_params(c))
        assert n == c["count"], c["source"]


def test_hash_kats(kats):
    for c in kats["hash"]:
        n, _, _ = oracle.kernel_execute(int(Operator.HashProbe), np.array(c["build"], dtype=np.uint64),
                                        kernel_params({"params": {}}), np.array(c["probe"], dtype=np.uint64))
        assert n == c["count"], c["source"]
        if "rows" in c:
            for key, rows in c["rows"].items():
                b = {"k": np.array(c["build"], dtype=np.int64)}
                p = {"k": np.array([int(key)], dtype=np.int64)}
                pr, br = oracle.join_pairs(p, None, "k", None, b, None, "k", None)
                assert sorted(br.tolist()) == rows


def test_join_table_kats(kats):
    for c in kats["join_tables"]:
        bk = gen_column(c["build_keys"], "i64")
        pk = gen_column(c["probe_keys"], "i64")
        extra = c.get("extra_probe_misses", [])
        pk = np.concatenate([pk, np.array(extra, dtype=np.int64)])
        pr, br = oracle.join_pairs({"k": pk}, None, "k", None, {"k": bk}, None, "k", None)
        nb = len(bk)
        assert np.array_equal(pr, np.arange(nb, dtype=np.uint32)), c["source"]
        assert np.array_equal(br, np.arange(nb, dtype=np.uint32)), c["source"]


def test_aggregate_kernel_kats(kats):
    for c in kats["aggregates"]:
        if c["op"] == "AggregateSumF64":
            v = np.array(c["f64"], dtype=np.float64) if "f64" in c else np.arange(c["f64_range"], dtype=np.float64)
            cnt, s, _ = oracle.kernel_execute(int(Operator.AggregateSumF64), v.view(np.uint64),
                                              kernel_params({"params": {}}))
            assert abs(s - c["sum"]) < 1e-9, c["source"]
        else:
            cnt, _, _ = oracle.kernel_execute(int(Operator.AggregateCountDistinct),
                                              np.array(c["cells"], dtype=np.uint64), kernel_params({"params": {}}))
            assert cnt == c["count"], c["source"]


def test_arithmetic_kats(kats):
    t = {k: np.array(v, dtype=np.int64) for k, v in kats["arithmetic"]["table"].items()}
    for c in kats["arithmetic"]["cases"]:
        out = oracle.aggregate(t, None, arith_aggs(c))
        assert sum(v.value for v in out.values[0]) == c["value"], c["source"]


def test_group_kats(kats):
    g = kats["groups"][0]
    t = {k: np.array(v, dtype=np.int64) for k, v in g["table"].items()}
    out = oracle.aggregate(t, None, [sum_(col("a")), count_star()], group_by=("grp",))
    got = [[k[0], v[0].value, v[1].value] for k, v in zip(out.keys, out.values)]
    assert got == g["groups"], g["source"]
    g = kats["groups"][1]
    t = {k: np.array(v, dtype=np.int64) for k, v in g["table"].items()}
    out = oracle.aggregate(t, None, [sum_(col("a")), count_star(), avg(col("b"))], group_by=("grp",))
    assert out.ngroups == g["ngroups"] and len(out.values[0]) == 3


def test_join_count_kats(kats):
    c = kats["join_counts"][0]
    left = {"id": np.array(c["left"], dtype=np.int64)}
    right = {"oid": np.array(c["right"], dtype=np.int64)}
    pr, br = oracle.join_pairs(left, None, "id", None, right, None, "oid", None)
    assert len(pr) == c["inner_rows"], c["source"]


def test_oracle_exact_int128_and_overflow_flag():
    # Sums past 2^63 stay exact; a wrapping per-row product raises the flag.
    big = np.full(4, 2**62, dtype=np.int64)
    out = oracle.aggregate({"a": big}, None, [sum_(col("a"))])
    assert out.values[0][0].value == 2**64
    out = oracle.aggregate({"a": big}, None, [sum_(col("a") * 4)])
    assert out.flags & A.RESULT_ROW_OVERFLOW


def test_reference_path_restatement_matches_oracle():
    """The timed CPU baseline computes the same answer as the exact oracle."""
    from oracle import refpath
    from turbogp_b200 import datagen, workloads
    tpl = workloads.selective_scan_sum()
    for n in [0, 1, 33, 2049, 300_001]:
        t = datagen.lineitem(n, seed=n)
        cols = {k: t[k] for k in ("ship_day", "discount_pct", "quantity", "price_cents")}
        r = refpath.selective_scan_sum(cols, tpl)
        o = oracle.aggregate(cols, refpath.COLTYPES, tpl.aggs, tpl.group_by, tpl.where)
        assert r["count"] == o.values[0][1].value
        assert int(r["sum"]) == o.values[0][0].value


def test_dispatch_kats(kats):
    """The reference's dispatcher tests over make_table(n) (src/engine/dispatch.rs)."""
    from turbogp_b200.engine import col, count_star, max_, sum_
    d = kats["dispatch"]
    assert d["table"] == {"id": "range", "val": {"mod": 20}, "grp": {"mod": 5}}
    for c in d["cases"]:
        n = c["n"]
        i = np.arange(n, dtype=np.uint64)
        t = {"id": i, "val": i % 20, "grp": i % 5}
        w = None
        if c["where"]:
            name, op, lit = c["where"]
            w = {"eq": col(name) == lit, "gt": col(name) > lit}[op]
        agg = c["agg"]
        if agg == "count_star":
            aggs = [count_star()]
        elif agg[0] == "sum":
            aggs = [sum_(col(agg[1]))]
        elif agg[0] == "max":
            aggs = [max_(col(agg[1]))]
        else:
            got = oracle.count_distinct(t[agg[1]])
            assert got == (c["value"], "exact"), c["source"]
            continue
        gb = (c["group_by"],) if "group_by" in c else ()
        out = oracle.aggregate(t, None, aggs, gb, w)
        if "ngroups" in c:
            keys = out.keys[:c.get("order_by_key_limit", len(out.keys))]
            assert len(keys) == c["ngroups"], c["source"]
            assert keys == sorted(keys)
        else:
            assert out.values[0][0].value == c["value"], c["source"]


def test_like_kats(kats):
    """LIKE on the string column: the reference's contains / prefix searches
    (src/exec/fm_index.rs tests) through the oracle's restatement of like()."""
    import numpy as np
    for k in kats["like"]:
        out = oracle.like(k["strings"], k["pattern"])
        if "expect" in k:
            bits = np.unpackbits(out.bitmap, bitorder="little")[:len(k["strings"])]
            assert bits.astype(bool).tolist() == k["expect"], k["source"]
        else:
            assert out.count == k["count"], k["source"]


def test_like_semantics_edge_cases():
    """like() details the reference's loop implies: '_' is one byte, '%' any
    run, a pattern '%' or '_' also matches itself literally first, trailing
    '%'s match the empty rest, the empty pattern matches only the empty
    string, NOT LIKE is the complement."""
    s = ["", "a", "ab", "abc", "a%c", "a_c", "xabcx", "aXc", "\u00e9t\u00e9"]
    # "a%c" LIKE 'a%' is false: the string's '%' equals the pattern's '%' and
    # is consumed literally before the wildcard is considered, leaving no
    # backtracking point (the reference's loop, expr.rs:2152-2158).
    cases = {"": [0], "%": list(range(9)), "a": [1], "a%": [1, 2, 3, 5, 7], "%c": [3, 4, 5, 7],
             "a_c": [3, 4, 5, 7], "a%%c": [3, 4, 5, 7], "%b%": [2, 3, 6], "_": [1], "__": [2],
             "a%c%": [3, 4, 5, 7], "%%": list(range(9)), "\u00e9%": [8], "_t%": [], "__t%": [8]}
    for p, want in cases.items():
        got = oracle.like(s, p)
        idx = [i for i in range(len(s)) if (got.bitmap[i >> 3] >> (i & 7)) & 1]
        assert idx == want, (p, idx, want)
        neg = oracle.like(s, p, negated=True)
        assert neg.count == len(s) - got.count
