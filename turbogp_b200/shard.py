"""Row sharding across ranks (one process per GPU) and the exact merge of
per-rank partial aggregates.

Rows are independent on this path, so a table is range-partitioned by row and
each rank aggregates its own shard; the only exchange is the merge of partial
results. Partials are exact (int128 sums as Python ints, u64 counts), so the
merge is exact: counts and SUM/AVG sums add, MIN/MAX take the extreme, and the
f64 view is recomputed from the merged exact value (AVG = sum / count).

``exchange_partials`` carries the partial integers as int64 limbs through
``torch.distributed.all_gather`` (NCCL on GPUs, gloo on CPU); groups are
matched by key tuple after the gather, and every rank ends with the whole
result. ``repartition_partials`` is the exchange for high-cardinality
results: each rank sends every group to the rank its key hashes to (one
``all_to_all_single``), and each rank merges, vectorised, the groups it owns,
so the result ends partitioned by key across the ranks.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import _capi as A
from .engine import Agg, AggResult, QueryOutput


def row_shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) rows of rank `rank`: contiguous, sizes differing by at most one."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def merge_outputs(outs: Sequence[QueryOutput], aggs: Sequence[Agg]) -> QueryOutput:
    """Exact merge of partial results of the same query over disjoint row sets."""
    groups: dict[tuple, list] = {}
    scanned = selected = flags = 0
    for o in outs:
        scanned += o.rows_scanned
        selected += o.rows_selected
        flags |= o.flags
        for key, vals in zip(o.keys, o.values):
            cur = groups.get(key)
            if cur is None:
                groups[key] = [AggResult(v.value, v.count, v.as_f64) for v in vals]
                continue
            for i, (a, v) in enumerate(zip(aggs, vals)):
                c = cur[i]
                if a.func in (A.AGG_MIN, A.AGG_MAX):
                    if v.count:
                        pick = min if a.func == A.AGG_MIN else max
                        c.value = pick(c.value, v.value) if c.count else v.value
                else:
                    c.value += v.value
                c.count += v.count
    keys = sorted(groups)
    values = []
    for k in keys:
        row = groups[k]
        for a, r in zip(aggs, row):
            if a.func == A.AGG_AVG:
                r.as_f64 = float(r.value) / r.count if r.count else 0.0
            else:
                r.as_f64 = float(r.value)
        values.append(row)
    if not outs or not any(o.keys for o in outs):
        # Scalar aggregate: exactly one group even when every shard is empty.
        if not keys and outs:
            keys, values = [()], [[AggResult(0, 0, 0.0) for _ in aggs]]
    return QueryOutput(keys, values, scanned, selected, flags)


_MASK64 = (1 << 64) - 1


def _encode(out: QueryOutput) -> np.ndarray:
    """[scanned, selected, flags, ngroups, nkeys, nagg, then per group: keys...,
    per aggregate (value lo, value hi, count)] as int64 words."""
    nk = len(out.keys[0]) if out.keys else 0
    na = len(out.values[0]) if out.values else 0
    words = [out.rows_scanned, out.rows_selected, out.flags, len(out.keys), nk, na]
    for key, vals in zip(out.keys, out.values):
        words.extend(key)
        for v in vals:
            words.extend([v.value & _MASK64, (v.value >> 64) & _MASK64, v.count])
    return np.array([w & _MASK64 for w in words], dtype=np.uint64).view(np.int64)


def _decode(a: np.ndarray) -> QueryOutput:
    w = [int(x) for x in a.view(np.uint64)]
    scanned, selected, flags, ng, nk, na = w[:6]
    pos, keys, values = 6, [], []
    for _ in range(ng):
        keys.append(tuple(int(np.int64(np.uint64(x))) for x in w[pos:pos + nk]))
        pos += nk
        row = []
        for _ in range(na):
            lo, hi, cnt = w[pos:pos + 3]
            pos += 3
            v = ((hi << 64) | lo)
            if v >= 1 << 127:
                v -= 1 << 128
            row.append(AggResult(v, cnt, float(v)))
        values.append(row)
    return QueryOutput(keys, values, scanned, selected, flags)


def exchange_partials(out: QueryOutput, aggs: Sequence[Agg], device=None, group=None) -> QueryOutput:
    """All ranks contribute their partial result; every rank returns the
    exact merged result (all_gather of the encoded partials)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    mine = torch.from_numpy(_encode(out))
    if device is not None:
        mine = mine.to(device)
    n = torch.tensor([mine.numel()], dtype=torch.int64, device=mine.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    cap = int(max(int(s.item()) for s in sizes))
    padded = torch.zeros(cap, dtype=torch.int64, device=mine.device)
    padded[:mine.numel()] = mine
    parts = [torch.zeros_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    outs = [_decode(p[:int(s.item())].cpu().numpy()) for p, s in zip(parts, sizes)]
    return merge_outputs(outs, aggs)


def key_owner(keys: np.ndarray, world: int) -> np.ndarray:
    """Rank owning each key tuple (rows of an int64 [g, k] array): splitmix64
    of the key words, chained, modulo the world size."""
    h = np.full(keys.shape[0], 0x9E3779B97F4A7C15, dtype=np.uint64)
    with np.errstate(over="ignore"):
        for j in range(keys.shape[1]):
            z = keys[:, j].view(np.uint64) ^ h
            z = z + np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            h = z ^ (z >> np.uint64(31))
    return (h % np.uint64(world)).astype(np.int64)


def _merge_rows(rows: np.ndarray, nk: int, na: int, funcs: Sequence[int]):
    """Combines received [keys | lo | hi | count] rows with equal keys: counts
    and sums add (int128 through 32-bit halves and a carry), MIN / MAX take the
    extreme. Returns (keys, lo, hi, count) sorted by key."""
    if rows.shape[0] == 0:
        z = np.zeros((0, na))
        return (np.zeros((0, nk), np.int64), z.astype(np.uint64), z.astype(np.int64), z.astype(np.uint64))
    keys = rows[:, :nk]
    order = np.lexsort(keys.T[::-1])
    rows = rows[order]
    keys = rows[:, :nk]
    lo = rows[:, nk:nk + na].view(np.uint64)
    hi = rows[:, nk + na:nk + 2 * na]
    cnt = rows[:, nk + 2 * na:nk + 3 * na].view(np.uint64)
    new = np.ones(rows.shape[0], dtype=bool)
    new[1:] = np.any(keys[1:] != keys[:-1], axis=1)
    starts = np.flatnonzero(new)
    out_lo = np.empty((starts.size, na), np.uint64)
    out_hi = np.empty((starts.size, na), np.int64)
    mask32 = np.uint64(0xFFFFFFFF)
    for a, f in enumerate(funcs):
        if f in (A.AGG_MIN, A.AGG_MAX):
            # Partials without rows for this aggregate do not take part (a
            # group whose partials all lack rows keeps its first value).
            v = lo[:, a].view(np.int64)
            ident = np.iinfo(np.int64).max if f == A.AGG_MIN else np.iinfo(np.int64).min
            has = cnt[:, a] > 0
            r = (np.minimum if f == A.AGG_MIN else np.maximum).reduceat(np.where(has, v, ident), starts)
            none = np.add.reduceat(has.astype(np.int64), starts) == 0
            r = np.where(none, v[starts], r)
            out_lo[:, a] = r.view(np.uint64)
            out_hi[:, a] = r >> 63
        else:
            s_ll = np.add.reduceat(lo[:, a] & mask32, starts)
            s_lh = np.add.reduceat(lo[:, a] >> np.uint64(32), starts)
            s_hi = np.add.reduceat(hi[:, a], starts)
            s_lh = s_lh + (s_ll >> np.uint64(32))
            out_lo[:, a] = ((s_lh & mask32) << np.uint64(32)) | (s_ll & mask32)
            out_hi[:, a] = s_hi + (s_lh >> np.uint64(32)).astype(np.int64)
    out_cnt = np.add.reduceat(cnt, starts, axis=0)
    return keys[starts], out_lo, out_hi, out_cnt


def repartition_partials(out: QueryOutput, aggs: Sequence[Agg], nkeys: int, device=None,
                         group=None) -> QueryOutput:
    """Hash-partitioned exact merge of a grouped partial result: every rank
    passes its partial (any number of groups, ``nkeys`` >= 1 key columns) and
    returns the merged groups whose key it owns (``key_owner``), sorted by key.
    The union over the ranks is the merged result of all partials; rows
    scanned / selected are the totals and flags the OR over the ranks."""
    import torch
    import torch.distributed as dist
    if nkeys < 1:
        raise ValueError("repartition needs a key; scalar results merge with exchange_partials")
    world = dist.get_world_size(group)
    na = len(aggs)
    keys, lo, hi, cnt = out.arrays()
    keys = keys.reshape(-1, nkeys)
    dest = key_owner(keys, world)
    rows = np.concatenate([keys, lo.view(np.int64), hi, cnt.view(np.int64)], axis=1) if keys.shape[0] else \
        np.zeros((0, nkeys + 3 * na), np.int64)
    order = np.argsort(dest, kind="stable")
    rows = np.ascontiguousarray(rows[order])
    width = nkeys + 3 * na
    send_counts = np.bincount(dest, minlength=world).astype(np.int64) * width
    dev = device if device is not None else torch.device("cpu")
    sc = torch.from_numpy(send_counts).to(dev)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    recv_counts = rc.cpu().numpy()
    send = torch.from_numpy(rows.reshape(-1)).to(dev)
    recv = torch.empty(int(recv_counts.sum()), dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv, send, output_split_sizes=[int(x) for x in recv_counts],
                           input_split_sizes=[int(x) for x in send_counts], group=group)
    meta = torch.tensor([out.rows_scanned, out.rows_selected, out.flags], dtype=torch.int64, device=dev)
    metas = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    metas = [m.cpu().numpy() for m in metas]
    k, mlo, mhi, mcnt = _merge_rows(recv.cpu().numpy().reshape(-1, width), nkeys, na, [a.func for a in aggs])
    ng = k.shape[0]
    vals = np.zeros(ng * na, dtype=[("lo", "<u8"), ("hi", "<i8"), ("count", "<u8"), ("as_f64", "<f8")])
    vals["lo"], vals["hi"], vals["count"] = mlo.reshape(-1), mhi.reshape(-1), mcnt.reshape(-1)
    # f64 views: the correctly rounded value (int64-representable values
    # convert exactly-rounded in numpy; wider ones through Python ints); AVG
    # divides by the merged count.
    small = (mhi.reshape(-1) == (mlo.reshape(-1).view(np.int64) >> 63))
    f = mlo.reshape(-1).view(np.int64).astype(np.float64)
    for i in np.flatnonzero(~small):
        f[i] = float((int(mhi.reshape(-1)[i]) << 64) | int(mlo.reshape(-1)[i]))
    funcs = np.tile(np.array([a.func for a in aggs]), ng)
    c = mcnt.reshape(-1).astype(np.float64)
    avg = funcs == A.AGG_AVG
    f[avg] = np.where(c[avg] > 0, f[avg] / np.where(c[avg] > 0, c[avg], 1.0), 0.0)
    vals["as_f64"] = f
    scanned = int(sum(int(m[0]) for m in metas))
    selected = int(sum(int(m[1]) for m in metas))
    flags = 0
    for m in metas:
        flags |= int(m[2])
    return QueryOutput(None, None, scanned, selected, flags,
                       raw=(np.ascontiguousarray(k).reshape(-1).view(np.uint64), vals, ng, nkeys, na))
