"""The reference's known answers through the C ABI on the GPU."""
import ctypes as C

import numpy as np
import pytest

from conftest import gen_column
from kat_helpers import arith_aggs, kernel_params, leaf, scalar_expect
from turbogp_b200.engine import avg, col, count_star, sum_
from turbogp_b200.kernel_table import KernelParams, KernelTable, MemoryTier, Operator, CpuTarget
import oracle

pytestmark = pytest.mark.gpu


def bits_of(bm, n):
    return np.unpackbits(bm, bitorder="little")[:n].astype(bool)


def test_filter_kats(ctx, kats):
    for c in kats["filters"]:
        x = gen_column(c["column"], c["dtype"])
        t = ctx.register({"c": x}, {"c": c["coltype"]})
        out = t.filter(leaf("c", c["cmp"], c["lit"]))
        if c["expect"] == "scalar":
            exp = scalar_expect(x, c["cmp"], c["lit"])
            assert np.array_equal(bits_of(out.bitmap, len(x)), exp), c["source"]
        elif isinstance(c["expect"], list):
            assert bits_of(out.bitmap, len(x)).tolist() == c["expect"], c["source"]
        else:
            assert out.count == c["expect"], c["source"]
        assert np.array_equal(out.rowids, np.flatnonzero(bits_of(out.bitmap, len(x))).astype(np.uint32))
        t.drop()


def test_conjunction_kats(ctx, kats):
    for c in kats["conjunctions"]:
        x = gen_column(c["column"], c["dtype"])
        t = ctx.register({"c": x}, {"c": c["coltype"]})
        (o1, v1), (o2, v2) = c["leaves"]
        assert t.filter(leaf("c", o1, v1) & leaf("c", o2, v2)).count == c["count"], c["source"]
        t.drop()


def test_kernel_table_registers_gpu_kernels(ctx):
    kt = KernelTable(ctx)
    assert len(kt.list()) == 7
    k = kt.select(Operator.ScanEqU64, MemoryTier.Hbm)
    assert k is not None and k.cpu() == CpuTarget.GpuSm100a
    # Fallback order of src/kernel/mod.rs:209-221: another tier still finds the GPU kernel.
    assert kt.select(Operator.ScanEqU64, MemoryTier.L3) is k
    assert kt.select(Operator.LeapfrogJoin, MemoryTier.Hbm) is None


def test_scan_kernel_kats(ctx, kats):
    kt = KernelTable(ctx)
    for c in kats["scan_kernels"]:
        cells = gen_column(c["cells"], "u64")
        p = kernel_params(c)
        p.cell_count = len(cells)
        out = np.zeros(64, dtype=np.uint8)
        r = kt.select(Operator[c["op"]], MemoryTier.Hbm).execute(cells.ctypes.data if len(cells) else 0,
                                                                 out.ctypes.data, p)
        assert r.count == c["count"], c["source"]
        oc, _, om = oracle.kernel_execute(int(Operator[c["op"]]), cells, kernel_params(c))
        assert r.mask == om, c["source"]


def test_hash_kernel_kats(ctx, kats):
    kt = KernelTable(ctx)
    build_k = kt.select(Operator.HashBuild, MemoryTier.Hbm)
    probe_k = kt.select(Operator.HashProbe, MemoryTier.Hbm)
    for c in kats["hash"]:
        keys = np.array(c["build"], dtype=np.uint64)
        out = np.zeros(64, dtype=np.uint8)
        r = build_k.execute(keys.ctypes.data, out.ctypes.data, KernelParams(cell_count=len(keys)))
        assert r.count == len(keys)
        handle = int(out[:8].view(np.uint64)[0])
        probe = np.concatenate([np.array([handle], dtype=np.uint64), np.array(c["probe"], dtype=np.uint64)])
        r = probe_k.execute(probe.ctypes.data, out.ctypes.data, KernelParams(cell_count=len(c["probe"])))
        assert r.count == c["count"], c["source"]
        ctx.hash_table_free(handle)


def test_aggregate_kernel_kats(ctx, kats):
    kt = KernelTable(ctx)
    for c in kats["aggregates"]:
        if c["op"] == "AggregateSumF64":
            v = np.array(c["f64"], dtype=np.float64) if "f64" in c else np.arange(c["f64_range"], dtype=np.float64)
            r = kt.select(Operator.AggregateSumF64, MemoryTier.Hbm).execute(v.ctypes.data, None,
                                                                           KernelParams(cell_count=len(v)))
            assert abs(r.sum - c["sum"]) <= 1e-12 * abs(c["sum"]), c["source"]
        else:
            v = np.array(c["cells"], dtype=np.uint64)
            r = kt.select(Operator.AggregateCountDistinct, MemoryTier.Hbm).execute(v.ctypes.data, None,
                                                                                  KernelParams(cell_count=len(v)))
            assert r.count == c["count"], c["source"]


def test_join_table_kats(ctx, kats):
    for c in kats["join_tables"]:
        bk = gen_column(c["build_keys"], "i64")
        pk = np.concatenate([gen_column(c["probe_keys"], "i64"), np.array(c.get("extra_probe_misses", []),
                                                                           dtype=np.int64)])
        b = ctx.register({"k": bk})
        p = ctx.register({"k": pk})
        j = b.join_build("k")
        pr, br = j.probe_pairs(p, "k")
        n = len(bk)
        assert np.array_equal(pr, np.arange(n, dtype=np.uint32)), c["source"]
        assert np.array_equal(br, np.arange(n, dtype=np.uint32)), c["source"]
        j.drop(); b.drop(); p.drop()


def test_arithmetic_group_join_kats(ctx, kats):
    t = ctx.register({k: np.array(v, dtype=np.int64) for k, v in kats["arithmetic"]["table"].items()})
    for c in kats["arithmetic"]["cases"]:
        out = t.aggregate(arith_aggs(c))
        assert sum(v.value for v in out.values[0]) == c["value"], c["source"]
    g = kats["groups"][0]
    t = ctx.register({k: np.array(v, dtype=np.int64) for k, v in g["table"].items()})
    out = t.aggregate([sum_(col("a")), count_star()], group_by=("grp",))
    assert [[k[0], v[0].value, v[1].value] for k, v in zip(out.keys, out.values)] == g["groups"]
    c = kats["join_counts"][0]
    left = ctx.register({"id": np.array(c["left"], dtype=np.int64)})
    right = ctx.register({"oid": np.array(c["right"], dtype=np.int64)})
    pr, br = right.join_build("oid").probe_pairs(left, "id")
    assert len(pr) == c["inner_rows"]
