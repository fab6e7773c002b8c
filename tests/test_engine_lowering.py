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
