"""tgp_aggregate_noalloc: the aggregate for callers that cannot allocate GPU
memory (an engine whose own allocator reserved the whole device, a serving
thread that may not take an allocation's device-wide synchronisation, a host
that forbids allocation after start-up). It must return what tgp_execute
returns for the same query, call after call, on the default stream and on a
stream of the caller's, in each accumulator placement (per-thread private,
per-CTA shared, global), while keeping all of its scratch in the library's
fixed 1 MiB device array.

This file is named so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

from turbogp_b200 import _capi as A
from turbogp_b200 import datagen, workloads
from turbogp_b200.engine import Context, Schema, col, count_star, sum_

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES


def noalloc(lib, dev_cols: dict, schema: Schema, aggs, domains, where, stream=None):
    """Calls the entry point through the C ABI. domains: [(name, min, count)];
    stream: a cudaStream_t handle (None = the default stream)."""
    names = schema.names
    descs = (A.ColumnDesc * len(names))()
    for i, n in enumerate(names):
        descs[i].dtype, descs[i].coltype, descs[i].data = schema.dtypes[i][0], schema.dtypes[i][1], dev_cols[n].data_ptr()
    nodes, npred = schema.lower_pred(where)
    q, keep = schema.lower_query(aggs, (), where)
    doms = (A.KeyDomain * max(1, len(domains)))()
    ngroups = 1
    for i, (n, lo, cnt) in enumerate(domains):
        doms[i].column, doms[i].min, doms[i].count = schema.index(n), lo, cnt
        ngroups *= cnt
    vals = (A.AggValue * (ngroups * len(aggs)))()
    res = A.QueryResult()
    msg = C.create_string_buffer(256)
    rows = dev_cols[names[0]].numel()
    st = lib.tgp_aggregate_noalloc(0, stream, descs, len(names), rows, nodes, npred, doms, len(domains), q.aggs,
                                   len(aggs), vals, ngroups * len(aggs), C.byref(res), msg, 256)
    return st, msg.value.decode(), vals, res, ngroups


def dense_index(key, domains):
    g = 0
    for v, (_, lo, cnt) in zip(key, domains):
        g = g * cnt + (v - lo)
    return g


def check_against_execute(expected, vals, res, ngroups, aggs, domains):
    assert res.rows_selected == expected.rows_selected
    assert res.ngroups == ngroups
    seen = set()
    for key, row in zip(expected.keys, expected.values):
        g = dense_index(key, domains)
        seen.add(g)
        for a, want in enumerate(row):
            got = vals[g * len(aggs) + a]
            assert got.value == want.value and got.count == want.count
            assert abs(got.as_f64 - want.as_f64) <= 1e-12 * abs(want.as_f64)
    for g in range(ngroups):
        if g not in seen:
            assert vals[g * len(aggs)].count == 0


# Per-thread private (scalar), per-CTA shared (6 flag groups x 6 slots) and
# global (2,526 ship days x 6 slots: too many for a CTA's shared memory)
# accumulator placements.
PLACEMENTS = [
    ("private", lambda: workloads.selective_scan_sum(), []),
    ("shared", lambda: workloads.filtered_group_agg(), [("flag_a", 0, 3), ("flag_b", 0, 2)]),
    ("global", lambda: workloads.filtered_group_agg(), [("ship_day", datagen.DAY0, datagen.NDAYS)]),
]


@pytest.mark.parametrize("rows", [1_000_003, 60_000])
def test_noalloc_matches_execute_on_two_calls_in_a_row(rows):
    import torch
    host = datagen.lineitem(rows, seed=17)
    dev = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    schema = Schema.of(host, CT)
    lib = A.load()
    with Context(0) as ctx:
        table = ctx.register(host, CT)
        for _, mk, domains in PLACEMENTS:
            tpl = mk()
            group_by = tuple(n for n, _, _ in domains)
            expected = table.aggregate(tpl.aggs, group_by, tpl.where)
            for _ in range(2):
                st, msg, vals, res, ngroups = noalloc(lib, dev, schema, tpl.aggs, domains, tpl.where)
                assert st == A.OK, msg
                check_against_execute(expected, vals, res, ngroups, tpl.aggs, domains)


def test_noalloc_on_a_caller_stream_keeps_the_current_device():
    import torch
    host = datagen.lineitem(300_007, seed=23)
    dev = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    schema = Schema.of(host, CT)
    lib = A.load()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with Context(0) as ctx:
        table = ctx.register(host, CT)
        for _, mk, domains in PLACEMENTS:
            tpl = mk()
            expected = table.aggregate(tpl.aggs, tuple(n for n, _, _ in domains), tpl.where)
            for _ in range(2):
                st, msg, vals, res, ngroups = noalloc(lib, dev, schema, tpl.aggs, domains, tpl.where,
                                                      stream=C.c_void_p(s.cuda_stream))
                assert st == A.OK, msg
                check_against_execute(expected, vals, res, ngroups, tpl.aggs, domains)
                assert torch.cuda.current_device() == 0


def test_noalloc_rejects_oversized_scratch_and_bad_domains():
    import torch
    host = datagen.lineitem(10_000, seed=3)
    dev = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    schema = Schema.of(host, CT)
    lib = A.load()
    aggs = workloads.filtered_group_agg().aggs
    # 2,526 ship days x 3 flags x (6 accumulators x 16 B + 6 results x 32 B) > 1 MiB.
    st, msg, *_ = noalloc(lib, dev, schema, aggs, [("ship_day", datagen.DAY0, datagen.NDAYS), ("flag_a", 0, 3)],
                          None)
    assert st == A.CAPACITY and "fixed maximum" in msg
    # flag_a holds 0..2: a domain of two values is rejected before any accumulation.
    st, msg, *_ = noalloc(lib, dev, schema, [count_star(), sum_(col("quantity"))], [("flag_a", 0, 2)], None)
    assert st == A.INVALID_ARG and "domain" in msg
    # The array is shared: a valid call right after the failures is still exact.
    st, msg, vals, res, _ = noalloc(lib, dev, schema, [count_star(), sum_(col("quantity"))], [("flag_a", 0, 3)], None)
    assert st == A.OK, msg
    for g in range(3):
        sel = host["flag_a"] == g
        assert vals[2 * g].value == int(sel.sum())
        assert vals[2 * g + 1].value == int(host["quantity"][sel].astype(np.int64).sum())
