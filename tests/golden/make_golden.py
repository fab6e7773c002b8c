"""Writes ``reference_kats.json``: the known-answer tests the reference's own
unit tests hold for the hot path, transcribed from its test sources (read as
text; the Rust reference cannot be built here). Each case names the test it
comes from (path inside pkhairkh/turboGP : line) and describes its input by a
generator formula, so the fixture stays small.

Generators: {"list": [...]}, {"range": [start, stop]} (stop exclusive),
{"mod": [n, m]} (i % m for i < n), {"rep": [v, n]}, {"f64_scaled": [n, k]}
((i as f64) * k), {"i32_mix": [n]} (((i * 7) % 51) - 25).

Run: python tests/golden/make_golden.py
"""
import json
from pathlib import Path

T = lambda s: [c == "T" for c in s]  # noqa: E731

BITMAP = "src/exec/bitmap.rs"
SCAN = "src/kernel/scan.rs"
HASH = "src/kernel/hash.rs"
AGG = "src/kernel/aggregate.rs"
JHT = "src/exec/join_hash_table.rs"
ARITH = "tests/arithmetic_aggregates.rs"
JOINS = "tests/joins_groupby_orderby.rs"
FM = "src/exec/fm_index.rs"

ten = {"list": [10, 20, 30, 40, 50, 60, 70, 80, 90, 100]}
fives = {"list": [1, 5, 5, 3, 5, 7, 8, 5, 9, 10]}
f5 = {"list": [1.0, 2.5, 2.5, 3.0, 2.5]}
f10 = {"list": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0, 9.0, 10.0]}
signed = {"list": [-5, -3, -1, 0, 1, 3, 5]}

filters = [
    # (source, dtype, coltype, column, cmp, literal, expected bits or count)
    (f"{BITMAP}:1126", "u64", "date", fives, "eq", 5, T("FTTFTFFTFF")),
    (f"{BITMAP}:1133", "u64", "date", ten, "lt", 50, T("TTTTFFFFFF")),
    (f"{BITMAP}:1140", "u64", "date", ten, "ge", 50, T("FFFFTTTTTT")),
    (f"{BITMAP}:1147", "u64", "date", ten, "le", 50, T("TTTTTFFFFF")),
    (f"{BITMAP}:1154", "u64", "date", ten, "gt", 50, T("FFFFFTTTTT")),
    (f"{BITMAP}:1161", "u64", "date", fives, "ne", 5, T("TFFTFTTFTT")),
    (f"{BITMAP}:1168", "f64", "float", f5, "ne", 2.5, T("TFFTF")),
    (f"{BITMAP}:1175", "f64", "float", f5, "eq", 2.5, T("FTTFT")),
    (f"{BITMAP}:1182", "f64", "float", f10, "lt", 5.0, T("TTTTFFFFFF")),
    (f"{BITMAP}:1192", "f64", "float", f10, "le", 5.0, T("TTTTTFFFFF")),
    (f"{BITMAP}:1202", "f64", "float", f10, "ge", 5.0, T("FFFFTTTTTT")),
    (f"{BITMAP}:1212", "f64", "float", f10, "gt", 5.0, T("FFFFFTTTTT")),
    (f"{BITMAP}:1222", "i64", "int", signed, "lt", 0, T("TTTFFFF")),
    (f"{BITMAP}:1230", "i64", "int", signed, "ge", 0, T("FFFTTTT")),
    (f"{BITMAP}:1257", "u64", "date", {"mod": [1_000_000, 100]}, "eq", 50, 10_000),
    (f"{BITMAP}:1265", "f64", "float", {"f64_scaled": [1_000_000, 0.001]}, "lt", 50.0, 50_000),
    (f"{BITMAP}:1388", "i32", "int", fives, "eq", 5, T("FTTFTFFTFF")),
    (f"{BITMAP}:1395", "i32", "int", {"list": [-5, -3, 0, 3, 5, 7, 9, 12, 15, 20]}, "lt", 5, T("TTTTFFFFFF")),
]
small_i32 = {"list": [-2, -1, 0, 1, 2, 3, 4, 5]}
for op, bits in [("eq", "FFFFTFFF"), ("ne", "TTTTFTTT"), ("lt", "TTTTFFFF"), ("le", "TTTTTFFF"),
                 ("gt", "FFFFFTTT"), ("ge", "FFFFTTTT")]:
    filters.append((f"{BITMAP}:1403", "i32", "int", small_i32, op, 2, T(bits)))

# test_filter_i32_avx512_vs_scalar (bitmap.rs:1417-1471): every op against the
# test's own scalar definition, for these literals.
i32_mix = {"i32_mix": [1000]}
mix_cases = [(f"{BITMAP}:1417", "i32", "int", i32_mix, op, v, "scalar")
             for v in [-100, -25, -1, 0, 7, 25, 100] for op in ["eq", "ne", "lt", "le", "gt", "ge"]]

conjunctions = [
    # bitmap.rs:1274 test_large_and_into_bool: 10 <= i%100 <= 50 over 1M rows.
    {"source": f"{BITMAP}:1274", "column": {"mod": [1_000_000, 100]}, "dtype": "u64", "coltype": "date",
     "leaves": [["ge", 10], ["le", 50]], "count": 410_000},
]

scan_kernels = [
    # (source, op, cells, params, expected count)
    (f"{SCAN}:641", "ScanEqU64", {"list": [1, 2, 3, 2, 4, 2, 5]}, {"target_u64": 2}, 3),
    (f"{SCAN}:648", "ScanRangeU64", {"list": [1, 5, 10, 15, 20, 25, 30]}, {"low_u64": 10, "high_u64": 20}, 3),
    (f"{SCAN}:677", "ScanEqU64", {"mod": [1000, 7]}, {"target_u64": 3}, 143),
    (f"{SCAN}:689", "ScanEqU64", {"mod": [10000, 7]}, {"target_u64": 3}, 1429),
    (f"{SCAN}:713", "ScanRangeU64", {"range": [0, 1000]}, {"low_u64": 100, "high_u64": 200}, 101),
    (f"{SCAN}:736", "ScanEqU64", {"list": []}, {"target_u64": 42}, 0),
    (f"{SCAN}:747", "ScanMultiPredicate", {"range": [0, 21]}, {"preds": [[5, "Eq"], [2, "Gt"], [10, "Lt"]]}, 1),
    (f"{SCAN}:757", "ScanMultiPredicate", {"rep": [5, 100]}, {"preds": [[5, "Eq"], [0, "Gt"], [100, "Lt"]]}, 100),
    (f"{SCAN}:767", "ScanMultiPredicate", {"range": [0, 1000]}, {"preds": [[1000, "Gt"], [1000, "Lt"], [5, "Eq"]]}, 0),
    (f"{SCAN}:776", "ScanMultiPredicate", {"list": []}, {"preds": [[5, "Eq"], [2, "Gt"], [10, "Lt"]]}, 0),
    (f"{SCAN}:784", "ScanMultiPredicate", {"range": [0, 100]}, {"preds": [[7, "Eq"]]}, 1),
    (f"{SCAN}:793", "ScanMultiPredicate", {"range": [0, 100]}, {"preds": [[50, "Gt"], [60, "Lt"]]}, 9),
    (f"{SCAN}:802", "ScanMultiPredicate", {"range": [0, 100]}, {"preds": [[10, "Gt"], [20, "Lt"]]}, 9),
    (f"{SCAN}:812", "ScanMultiPredicate", {"range": [0, 1000]}, {"preds": [[500, "Eq"], [100, "Gt"], [900, "Lt"]]}, 1),
    (f"{SCAN}:826", "ScanMultiPredicate", {"range": [0, 1234]}, {"preds": [[100, "Gt"], [200, "Lt"]]}, 99),
    (f"{SCAN}:839", "ScanMultiPredicate", {"mod": [1000, 17]}, {"preds": [[5, "Eq"]]}, 59),
    (f"{SCAN}:864", "ScanMultiPredicate", {"range": [0, 1000]}, {"preds": [[1000, "Gt"], [0, "Lt"], [5, "Eq"]]}, 0),
    (f"{SCAN}:876", "ScanMultiPredicate", {"rep": [5, 1000]}, {"preds": [[5, "Eq"], [0, "Gt"], [10, "Lt"]]}, 1000),
]

hash_kats = [
    # build keys, probe keys, expected matched pairs
    {"source": f"{HASH}:232", "build": [1, 2, 3, 2, 4, 2, 5], "probe": [2], "count": 3, "rows": {"2": [1, 3, 5]}},
    {"source": f"{HASH}:232", "build": [1, 2, 3, 2, 4, 2, 5], "probe": [99], "count": 0},
    {"source": f"{HASH}:247", "build": [1, 2, 3, 2, 4], "probe": [2, 4, 99], "count": 3},
    {"source": f"{JHT}:262", "build": [42, 42, 42], "probe": [42], "count": 3},
]
join_kats = [
    # join_hash_table.rs:248 insert i*7 -> row i (i < 100); probe(i*7) = i; probe 1, 999 miss.
    {"source": f"{JHT}:248", "build_keys": {"scaled": [100, 7]}, "probe_keys": {"scaled": [100, 7]},
     "extra_probe_misses": [1, 999], "pairs": "identity"},
    # join_hash_table.rs:276 100K keys i -> row i, then 1000 misses.
    {"source": f"{JHT}:276", "build_keys": {"range": [0, 100_000]}, "probe_keys": {"range": [0, 101_000]},
     "pairs": "identity_below", "below": 100_000},
]
agg_kats = [
    {"source": f"{AGG}:199", "op": "AggregateSumF64", "f64": [1.0, 2.0, 3.0, 4.0, 5.0], "sum": 15.0},
    {"source": f"{AGG}:219", "op": "AggregateSumF64", "f64_range": 100, "sum": 4950.0},
    {"source": f"{AGG}:230", "op": "AggregateCountDistinct", "cells": [1, 2, 3, 2, 4, 1, 5], "count": 5},
]
# Engine-level KATs: table (id, price, discount) = (1,100,10), (2,200,20), (3,300,30).
arith = {
    "table": {"id": [1, 2, 3], "price": [100, 200, 300], "discount": [10, 20, 30]},
    "cases": [
        {"source": f"{ARITH}:15", "sum_of": [[["price", 1, 0], [None, 0, 2]]], "value": 1200},
        {"source": f"{ARITH}:24", "sum_of": [[["price", 1, 0]], [["discount", 1, 0]]], "value": 660},
        {"source": f"{ARITH}:33", "sum_of": [[["price", 1, 0]], [["discount", -1, 0]]], "value": 540},
        {"source": f"{ARITH}:42", "sum_of": [[["price", 1, 0], [None, 0, 2]], [["discount", -1, 0], [None, 0, 2]]],
         "value": 1080},
        {"source": f"{ARITH}:51", "sum_of": [[["price", 1, 0], ["discount", 1, 0]]], "value": 14000},
        {"source": f"{ARITH}:60", "sum_of": [[["price", 1, 0]]], "value": 600},
        {"source": f"{ARITH}:68", "count_star": True, "value": 3},
    ],
}
group_kats = [
    {"source": f"{JOINS}:82", "table": {"grp": [1, 1, 1, 2, 2], "a": [10, 20, 30, 40, 50]},
     "groups": [[1, 60, 3], [2, 90, 2]]},
    {"source": f"{JOINS}:66", "table": {"grp": [1, 1, 2], "a": [10, 20, 30], "b": [100, 200, 300]},
     "ngroups": 2},
]
join_count_kats = [
    {"source": f"{JOINS}:36", "left": [1, 2, 3], "right": [1], "inner_rows": 1},
]
# execute_dispatched over make_table(n): id = i, val = i % 20, grp = i % 5
# (src/engine/dispatch.rs:1694-1720); the queries of its tests on this path.
DISPATCH = "src/engine/dispatch.rs"
dispatch_kats = {
    "table": {"id": "range", "val": {"mod": 20}, "grp": {"mod": 5}},
    "cases": [
        {"source": f"{DISPATCH}:1778", "n": 100, "agg": "count_star", "where": None, "value": 100},
        {"source": f"{DISPATCH}:1789", "n": 100, "agg": "count_star", "where": ["val", "eq", 5], "value": 5},
        {"source": f"{DISPATCH}:1800", "n": 100, "agg": ["sum", "val"], "where": ["val", "gt", 15],
         "value": 350},
        {"source": f"{DISPATCH}:1813", "n": 100, "agg": "count_star", "group_by": "grp", "where": None,
         "ngroups": 5},
        {"source": f"{DISPATCH}:1824", "n": 100, "agg": "count_star", "group_by": "grp", "where": None,
         "order_by_key_limit": 3, "ngroups": 3},
        {"source": f"{DISPATCH}:1838", "n": 100, "agg": ["max", "val"], "where": None, "value": 19},
        {"source": f"{DISPATCH}:1849", "n": 100, "agg": ["count_distinct", "val"], "where": None, "value": 20},
        {"source": f"{DISPATCH}:1885", "n": 1_000_000, "agg": "count_star", "where": ["val", "eq", 5],
         "value": 50000},
    ],
}

# StringSearchColumn's contains / prefix searches (src/exec/fm_index.rs
# tests), which are LIKE '%s%' and LIKE 's%' on the interpreter's path.
urls4 = ["https://google.com/search", "https://yahoo.com", "http://google.com/maps", "https://bing.com"]
urls3 = ["https://google.com", "http://yahoo.com", "https://bing.com"]
like_kats = [
    {"source": f"{FM}:576", "strings": ["google.com", "yahoo.com", "google Maps"], "pattern": "%google%",
     "expect": [True, False, True]},
    {"source": f"{FM}:551", "strings": urls4, "pattern": "%google%", "count": 2},
    {"source": f"{FM}:551", "strings": urls4, "pattern": "%yahoo%", "count": 1},
    {"source": f"{FM}:551", "strings": urls4, "pattern": "%duckduckgo%", "count": 0},
    {"source": f"{FM}:564", "strings": urls3, "pattern": "https://%", "count": 2},
    {"source": f"{FM}:564", "strings": urls3, "pattern": "http://%", "count": 1},
    {"source": f"{FM}:564", "strings": urls3, "pattern": "ftp://%", "count": 0},
]

out = {
    "filters": [dict(source=s, dtype=d, coltype=c, column=col, cmp=op, lit=v, expect=e)
                for s, d, c, col, op, v, e in filters + mix_cases],
    "conjunctions": conjunctions,
    "scan_kernels": [dict(source=s, op=o, cells=c, params=p, count=n) for s, o, c, p, n in scan_kernels],
    "hash": hash_kats,
    "join_tables": join_kats,
    "aggregates": agg_kats,
    "arithmetic": arith,
    "groups": group_kats,
    "join_counts": join_count_kats,
    "dispatch": dispatch_kats,
    "like": like_kats,
}
Path(__file__).with_name("reference_kats.json").write_text(json.dumps(out, indent=1) + "\n")
print("wrote", sum(len(v) if isinstance(v, list) else 1 for v in out.values()), "groups of cases")
