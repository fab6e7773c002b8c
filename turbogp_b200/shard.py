"""Row sharding across ranks (one process per GPU) and the exact merge of
per-rank partial aggregates.

Rows are independent on this path, so a table is range-partitioned by row and
each rank aggregates its own shard; the only exchange is the merge of partial
results. Partials are exact (int128 sums as Python ints, u64 counts), so the
merge is exact: counts and SUM/AVG sums add, MIN/MAX take the extreme, and the
f64 view is recomputed from the merged exact value (AVG = sum / count).

``exchange_partials`` carries the partial integers as int64 limbs through
``torch.distributed.all_gather`` (NCCL on GPUs, gloo on CPU); groups are
matched by key tuple after the gather.
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
