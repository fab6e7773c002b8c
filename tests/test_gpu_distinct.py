"""tgp_count_distinct against the oracle: the exact path below 100,000
selected rows and the HyperLogLog path above it give the reference's numbers
(the registers are exact, so the estimates agree bit for bit)."""
import numpy as np
import pytest

import oracle
from turbogp_b200 import datagen
from turbogp_b200.engine import col

pytestmark = pytest.mark.gpu


def cells_of(a: np.ndarray) -> np.ndarray:
    if a.dtype == np.float64:
        return a.view(np.uint64)
    if a.dtype == np.uint64:
        return a
    return a.astype(np.int64).view(np.uint64)  # the reference's cell of the value


@pytest.mark.parametrize("n", [0, 1, 99_999, 100_000, 1_000_003, 6_000_000])
def test_count_distinct_matches_oracle(ctx, n):
    rng = np.random.default_rng(n + 5)
    cols = {
        "u8": rng.integers(0, 256, n, dtype=np.uint8),
        "i32": rng.integers(-(2**31), 2**31, n, dtype=np.int64).astype(np.int32),
        "i64": datagen.zipf_ranks(n, 10_000_000, 1.1, rng) - 5_000_000 if n else np.zeros(0, np.int64),
        "f64": np.round(rng.normal(0, 1000, n), 1),
        "u64": rng.integers(0, 2**64 - 1, n, dtype=np.uint64),
        "sel": rng.integers(0, 100, n).astype(np.int32),
    }
    cts = {"u64": "date"}
    t = ctx.register(cols, cts)
    for where in [None, col("sel") < 50, col("sel") < 2]:
        if where is None:
            bm = None
        else:
            bm = oracle.filter(cols, cts, where).bitmap
        for name in ("u8", "i32", "i64", "f64", "u64"):
            got = t.count_distinct(name, where)
            want = oracle.count_distinct(cells_of(cols[name]), bm)
            assert got == want, (n, name, where is None)
    t.drop()


def test_threshold_on_selected_rows(ctx):
    n = 150_000
    rng = np.random.default_rng(8)
    cols = {"v": rng.integers(0, 60_000, n).astype(np.int64), "r": np.arange(n, dtype=np.int32)}
    t = ctx.register(cols)
    for k, method in [(99_999, "exact"), (100_000, "hll")]:
        w = col("r") < k
        got = t.count_distinct("v", w)
        assert got == oracle.count_distinct(cells_of(cols["v"]), oracle.filter(cols, None, w).bitmap)
        assert got[1] == method
    t.drop()
