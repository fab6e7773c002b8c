"""The oracle's COUNT(DISTINCT): its xxh3_64 restatement pinned against the
xxhash package, and its HyperLogLog against the reference's own tests
(src/exec/hll.rs:142-187) and thresholds (aggregate.rs:1308-1325)."""
import numpy as np
import xxhash

import oracle


def test_xxh3_matches_the_xxhash_package():
    rng = np.random.default_rng(1)
    vals = [0, 1, 42, 2**32 - 1, 2**32, 2**63, 2**64 - 1] + [int(x) for x in rng.integers(0, 2**64 - 1, 20_000,
                                                                                           dtype=np.uint64)]
    for v in vals:
        assert oracle.xxh3_u64(v) == xxhash.xxh3_64_intdigest(v.to_bytes(8, "little")), hex(v)


def test_hll_reference_tests():
    # test_hll_empty: an empty sketch estimates 0.
    assert oracle.hll_estimate(np.zeros(0, dtype=np.uint64)) == 0
    # test_hll_single: one value estimates 1 or 2.
    assert 1 <= oracle.hll_estimate(np.array([42], dtype=np.uint64)) <= 2
    # test_hll_small_exact: below 100,000 rows the count is exact.
    assert oracle.count_distinct(np.arange(1000, dtype=np.uint64)) == (1000, "exact")
    # test_hll_large_approximate: 1M distinct values within 2 %.
    c, m = oracle.count_distinct(np.arange(1_000_000, dtype=np.uint64))
    assert m == "hll" and abs(c - 1_000_000) / 1_000_000 < 0.02
    # test_hll_with_duplicates: 500K values twice within 2 %.
    col = np.concatenate([np.arange(500_000, dtype=np.uint64)] * 2)
    c, m = oracle.count_distinct(col)
    assert m == "hll" and abs(c - 500_000) / 500_000 < 0.02
    # test_hll_merge: registers are a max, so order and chunking do not matter.
    rng = np.random.default_rng(2)
    perm = rng.permutation(col)
    assert oracle.hll_estimate(perm) == oracle.hll_estimate(col)


def test_threshold_counts_selected_rows():
    rng = np.random.default_rng(3)
    cells = rng.integers(0, 50_000, 150_000).astype(np.uint64)
    sel = np.zeros(150_000, dtype=bool)
    sel[:99_999] = True
    bm = np.packbits(sel, bitorder="little")
    assert oracle.count_distinct(cells, bm) == (len(np.unique(cells[:99_999])), "exact")
    sel[99_999] = True
    bm = np.packbits(sel, bitorder="little")
    c, m = oracle.count_distinct(cells, bm)
    assert m == "hll" and abs(c - len(np.unique(cells[:100_000]))) / len(np.unique(cells[:100_000])) < 0.03


def test_library_estimator_matches_the_oracle():
    """The library's host-side estimate (tgp_hll_estimate, the arithmetic
    tgp_count_distinct applies to the device registers) equals the oracle's,
    in the linear-counting and in the raw regime."""
    import ctypes as C
    from turbogp_b200 import _capi as A
    lib = A.load()
    rng = np.random.default_rng(4)
    cases = [np.zeros(16384, np.uint32), np.full(16384, 65, np.uint32)]
    for zero_frac in (0.999, 0.9, 0.5, 0.1, 0.0):
        r = rng.geometric(0.5, 16384).astype(np.uint32)
        r[rng.random(16384) < zero_frac] = 0
        cases.append(r)
    for regs in cases:
        out = C.c_uint64()
        assert lib.tgp_hll_estimate(regs.ctypes.data, C.byref(out)) == A.OK
        assert out.value == oracle._lib().orc_hll_estimate_regs(regs.ctypes.data)
