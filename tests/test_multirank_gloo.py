"""Row shards over two gloo ranks on the CPU: each rank aggregates its shard
with the oracle (standing in for its GPU), the partials are exchanged with
all_gather and merged exactly; the result equals the whole-table oracle."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle
from turbogp_b200 import datagen, shard, workloads
from turbogp_b200.engine import avg, col, count_star, max_, min_, sum_


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _same(a, b):
    assert a.keys == b.keys and a.rows_selected == b.rows_selected and a.rows_scanned == b.rows_scanned
    for ga, gb in zip(a.values, b.values):
        for x, y in zip(ga, gb):
            assert (x.value, x.count) == (y.value, y.count)
            assert abs(x.as_f64 - y.as_f64) <= 1e-12 * max(1.0, abs(y.as_f64))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 50_003
        full = datagen.lineitem(n, seed=77)
        lo, hi = shard.row_shard(n, rank, world)
        mine = {k: v[lo:hi] for k, v in full.items()}
        CT = datagen.LINEITEM_COLTYPES
        cases = [workloads.filtered_group_agg(), workloads.selective_scan_sum()]
        extra = workloads.filtered_group_agg()
        extra.aggs = [count_star(), min_(col("price_cents")), max_(col("quantity") - 60), avg(col("tax_pct")),
                      sum_(col("price_cents") * col("price_cents"))]
        cases.append(extra)
        empty = workloads.selective_scan_sum(days=1, qty_lt=1)       # nothing passes
        cases.append(empty)
        for tpl in cases:
            part = oracle.aggregate(mine, CT, tpl.aggs, tpl.group_by, tpl.where)
            merged = shard.exchange_partials(part, tpl.aggs)
            _same(merged, oracle.aggregate(full, CT, tpl.aggs, tpl.group_by, tpl.where))
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent, which fails the test
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_row_shard_partition():
    for n in [0, 1, 7, 100, 50_003]:
        for world in [1, 2, 3, 8]:
            parts = [shard.row_shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [h - l for l, h in parts]
            assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_merge_exactly():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: "ok", 1: "ok"}, res


def _rank_repartition(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 60_000
        rng = np.random.default_rng(5)
        full = {"key": datagen.zipf_ranks(n, 30_000, 1.1, rng) * 1_000_003 - 2**40,   # signed, sparse
                "g2": rng.integers(0, 4, n).astype(np.int32),
                "v": rng.integers(-1000, 1001, n).astype(np.int32),
                "w": rng.integers(0, 2**62, n, dtype=np.int64)}                      # int128 sums
        lo, hi = shard.row_shard(n, rank, world)
        mine = {k: v[lo:hi] for k, v in full.items()}
        aggs = [count_star(), sum_(col("v")), min_(col("v")), max_(col("w")), avg(col("v")), sum_(col("w"))]
        for gb, where in [(("key",), None), (("key", "g2"), col("v") > -500)]:
            part = oracle.aggregate(mine, None, aggs, gb, where)
            got = shard.repartition_partials(part, aggs, len(gb))
            want = oracle.aggregate(full, None, aggs, gb, where)
            owner = shard.key_owner(np.array(want.keys, dtype=np.int64).reshape(-1, len(gb)), world)
            keep = [i for i in range(len(want.keys)) if owner[i] == rank]
            assert got.keys == [want.keys[i] for i in keep]
            assert got.rows_scanned == want.rows_scanned and got.rows_selected == want.rows_selected
            for i, row in zip(keep, got.values):
                for x, y in zip(row, want.values[i]):
                    assert (x.value, x.count) == (y.value, y.count)
                    assert abs(x.as_f64 - y.as_f64) <= 1e-12 * max(1.0, abs(y.as_f64))
            # Every group lands on exactly one rank.
            sizes = [None] * world
            dist.all_gather_object(sizes, len(got.keys))
            assert sum(sizes) == len(want.keys)
        # Two rows over three ranks: one rank contributes no group at all.
        tiny = {k: v[:2] for k, v in full.items()}
        lo, hi = shard.row_shard(2, rank, world)
        part = oracle.aggregate({k: v[lo:hi] for k, v in tiny.items()}, None, aggs, ("key",), None)
        got = shard.repartition_partials(part, aggs, 1)
        want = oracle.aggregate(tiny, None, aggs, ("key",), None)
        owner = shard.key_owner(np.array(want.keys, dtype=np.int64).reshape(-1, 1), world)
        assert got.keys == [k for k, o in zip(want.keys, owner) if o == rank]
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent, which fails the test
        import traceback
        q.put((rank, traceback.format_exc()))
    finally:
        dist.destroy_process_group()


def test_repartitioned_merge_over_three_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_repartition, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: "ok", 1: "ok", 2: "ok"}, res
