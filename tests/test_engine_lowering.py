"""Host-side lowering of WHERE trees and the shard helpers, on the CPU."""
import numpy as np
import pytest
import xxhash

from turbogp_b200 import _capi as A
from turbogp_b200 import shard
from turbogp_b200.engine import Schema, col, string_cell


def test_string_literals_lower_to_their_hash():
    sc = Schema(["name", "q"], [(A.DT_U64, A.CT_INT), (A.DT_I32, A.CT_INT)])
    nodes, n = sc.lower_pred((col("name") == "banana") & (col("name") != "") & (col("q") < 5))
    assert n == 5
    assert nodes[0].lit == xxhash.xxh3_64_intdigest(b"banana") == string_cell("banana")
    assert nodes[1].lit == xxhash.xxh3_64_intdigest(b"") and nodes[1].cmp == A.CMP_NE
    assert nodes[3].lit == 5
    for bad in (col("name") < "m", col("name").between("a", "z")):
        with pytest.raises(ValueError):
            sc.lower_pred(bad)


def test_key_owner_is_deterministic_and_spread():
    keys = np.arange(-50_000, 50_000, dtype=np.int64).reshape(-1, 1)
    for world in (1, 2, 3, 8):
        a = shard.key_owner(keys, world)
        assert np.array_equal(a, shard.key_owner(keys.copy(), world))
        assert a.min() >= 0 and a.max() < world
        counts = np.bincount(a, minlength=world)
        assert counts.min() > 0.9 * len(keys) / world
    # Multi-column keys: every column takes part.
    k2 = np.stack([np.zeros(1000, np.int64), np.arange(1000, dtype=np.int64)], axis=1)
    assert len(set(shard.key_owner(k2, 8).tolist())) == 8


def test_merge_rows_int128_carries_and_empty_minmax():
    from turbogp_b200.engine import count_star, max_, min_, sum_, col
    aggs = [count_star(), sum_(col("v")), min_(col("v")), max_(col("v"))]
    funcs = [a.func for a in aggs]
    M = (1 << 64) - 1

    def row(key, total, count, mn, mx, mcount):
        vals = [(count, count), (total, count), (mn, mcount), (mx, mcount)]
        lo = [v & M for v, _ in vals]
        hi = [v >> 64 for v, _ in vals]
        cnt = [c for _, c in vals]
        return [key] + [int(np.uint64(x).view(np.int64)) for x in lo] + hi + cnt

    big = (1 << 100) + 12345          # needs the high limb
    rows = np.array([row(7, big, 3, -5, 9, 3), row(7, big, 2, -8, 4, 2), row(7, -3, 1, 0, 0, 0),
                     row(-1, (1 << 64) - 1, 1, 2, 2, 1), row(-1, 1, 1, 1, 1, 1)], dtype=np.int64)
    keys, lo, hi, cnt = shard._merge_rows(rows, 1, 4, funcs)
    assert keys.tolist() == [[-1], [7]]
    val = lambda g, a: (int(hi[g, a]) << 64) | int(lo[g, a])   # noqa: E731
    assert val(0, 1) == 1 << 64 and val(1, 1) == 2 * big - 3     # carries out of the low limb
    assert cnt[1].tolist() == [6, 6, 5, 5]
    assert int(lo[1, 2].view(np.int64)) == -8 and int(lo[1, 3].view(np.int64)) == 9   # the row without rows skipped
    assert int(lo[0, 2].view(np.int64)) == 1 and int(lo[0, 3].view(np.int64)) == 2
