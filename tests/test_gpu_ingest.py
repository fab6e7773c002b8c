"""tgp_table_register_cells: tables given in the reference's u64-cell layout,
narrowed on the device, answer every query exactly as the cells would."""
import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

import oracle
from turbogp_b200 import _capi as A
from turbogp_b200 import datagen, ingest, workloads
from turbogp_b200.engine import col, count_star, max_, min_, sum_

from test_gpu_parity import bits, predicates, same_query

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES
WANT = {"ship_day": A.DT_I32, "discount_pct": A.DT_U8, "quantity": A.DT_U8, "tax_pct": A.DT_U8,
        "price_cents": A.DT_I32, "flag_a": A.DT_U8, "flag_b": A.DT_U8}


def cells_of(host):
    return {k: v.astype(np.int64).view(np.uint64) for k, v in host.items()}


def check_lineitem(t, host, n):
    for i, p in enumerate(predicates()):
        g, o = t.filter(p), oracle.filter(host, CT, p)
        assert g.count == o.count and np.array_equal(bits(g.bitmap, n), bits(o.bitmap, n)), i
    for tpl in (workloads.filtered_group_agg(), workloads.selective_scan_sum()):
        same_query(t.aggregate(tpl.aggs, tpl.group_by, tpl.where), oracle.aggregate(host, CT, tpl.aggs, tpl.group_by,
                                                                                     tpl.where))


@pytest.mark.parametrize("n", [0, 1, 2049, 100_003])
def test_cells_narrow_and_match(ctx, n):
    host = datagen.lineitem(n, seed=41 + n)
    t = ctx.register_cells(cells_of(host), CT)
    if n:
        assert {k: dt for k, (dt, _) in zip(t.names, t.dtypes)} == WANT
    check_lineitem(t, host, n)
    t.drop()
    # i32 sidecars (as the reference's CSV loader keeps them) are taken as is.
    side = {k: v.astype(np.int32) for k, v in host.items() if k in ("ship_day", "quantity")}
    t = ctx.register_cells(cells_of(host), CT, side)
    assert t.dtypes[t.index("ship_day")][0] == A.DT_I32 and t.dtypes[t.index("quantity")][0] == A.DT_I32
    check_lineitem(t, host, n)
    t.drop()


def test_cells_that_do_not_narrow(ctx):
    rng = np.random.default_rng(12)
    n = 50_000
    raw = {
        "small_neg": rng.integers(-5, 6, n).astype(np.int64).view(np.uint64),         # Int -> I32
        "wide": rng.integers(-(2**40), 2**40, n).astype(np.int64).view(np.uint64),   # Int -> I64
        "date_hi": rng.integers(0, 2**64 - 1, n, dtype=np.uint64),                    # Date, cells >= 2^63 -> U64
        "date_small": rng.integers(0, 200, n).astype(np.uint64),                       # Date -> U8
        "f": rng.normal(0, 1e6, n).view(np.uint64),                                    # Float -> F64 bits
    }
    cts = {"small_neg": "int", "wide": "int", "date_hi": "date", "date_small": "date", "f": "float"}
    t = ctx.register_cells(raw, cts)
    got = {k: dt for k, (dt, _) in zip(t.names, t.dtypes)}
    assert got == {"small_neg": A.DT_I32, "wide": A.DT_I64, "date_hi": A.DT_U64, "date_small": A.DT_U8,
                   "f": A.DT_F64}
    # The oracle reads the raw cells (u64 words) with the same coltypes.
    host = {k: (v.view(np.float64) if k == "f" else v) for k, v in raw.items()}
    c = col
    preds = [c("small_neg") < 0, c("small_neg") >= -2, c("wide") > 2**39, c("wide").between(-(2**30), 2**30),
             c("date_hi") >= 2**63, c("date_hi") < 2**62, c("date_small") <= 100, (c("f") > 0.5) | (c("f") < -2e6),
             c("small_neg") == 3]
    for i, p in enumerate(preds):
        g, o = t.filter(p), oracle.filter(host, cts, p)
        assert g.count == o.count and np.array_equal(bits(g.bitmap, n), bits(o.bitmap, n)), i
    aggs = [count_star(), sum_(c("small_neg")), sum_(c("wide") * 3), min_(c("wide")), max_(c("small_neg"))]
    for gb in [(), ("small_neg",), ("date_small",)]:
        same_query(t.aggregate(aggs, gb, c("date_small") < 150, group_cap=1024),
                   oracle.aggregate(host, cts, aggs, gb, c("date_small") < 150))
    t.drop()


def test_parquet_to_hbm(ctx, tmp_path):
    host = datagen.lineitem(80_000, seed=43)
    arrow = pa.table({k: pa.array(v) for k, v in host.items()})
    p = tmp_path / "lineitem.parquet"
    pq.write_table(arrow, p)
    t = ingest.register_parquet(ctx, p, coltypes={"ship_day": "date"})
    check_lineitem(t, host, 80_000)
    t.drop()


def test_string_columns_compare_by_hash(ctx, tmp_path):
    rng = np.random.default_rng(17)
    words = np.array(["apple", "banana", "cherry", "", "ünïcødé", "x" * 40])
    n = 120_000
    pick = rng.integers(0, len(words), n)
    s = [None if i % 97 == 0 else str(words[k]) for i, k in enumerate(pick)]
    qty = rng.integers(1, 51, n).astype(np.int32)
    p = tmp_path / "strings.parquet"
    pq.write_table(pa.table({"name": pa.array(s, pa.string()), "quantity": pa.array(qty)}), p)
    t = ingest.register_parquet(ctx, p)
    cells, _, cts = ingest.read_parquet(p)
    host = {"name": cells["name"], "quantity": qty}
    c = col
    for where in [c("name") == "banana", c("name") != "cherry", (c("name") == "") & (c("quantity") < 10),
                  c("name") == "not there", c("name") == "x" * 40]:
        g, o = t.filter(where), oracle.filter(host, {"name": "int", "quantity": "int"}, where)
        assert g.count == o.count and np.array_equal(bits(g.bitmap, n), bits(o.bitmap, n))
    assert t.filter(c("name") == "banana").count == sum(1 for x in s if x == "banana")
    with pytest.raises(ValueError):
        t.filter(c("name") < "m")
    aggs = [count_star(), sum_(c("quantity"))]
    same_query(t.aggregate(aggs, ("name",), None, group_cap=64),
               oracle.aggregate(host, {"name": "int", "quantity": "int"}, aggs, ("name",), None))
    t.drop()
