"""Seeded synthetic tables with the distributions of the benchmark workloads.

TPC-H / ClickBench data are not available, so these tables stand in for them
with the stated shapes (one independent numpy PCG64 stream per column):

* ``lineitem(n)`` — the fact table of the filtered-aggregate and scan workloads:
  quantity i32 U[1,50], price_cents i64 U[90_000, 10_500_000], discount_pct
  i32 U[0,10], tax_pct i32 U[0,8], ship_day i32 uniform over 2,526
  consecutive days, flag_a u8 U{0,1,2}, flag_b u8 U{0,1}.
* ``dimension(n)`` — key i32 = seeded permutation of 1..n, order_day i32 over
  2,526 days, segment u8 U{0..24}.
* ``fact_fk(n, nkeys, s)`` — lineitem columns plus fk i32 drawn Zipf(s) over
  the keys 1..nkeys (inverse-CDF table).
* ``highcard(n, nkeys, s)`` — key i64 Zipf(s) over nkeys values, value i32
  U[0,1000].
"""
from __future__ import annotations

import os
import zlib
from concurrent.futures import ThreadPoolExecutor

import numpy as np

DAY0 = 8035          # 1992-01-01 as days since 1970-01-01
NDAYS = 2526
LINEITEM_COLTYPES = {"quantity": "int", "price_cents": "int", "discount_pct": "int", "tax_pct": "int",
                     "ship_day": "date", "flag_a": "int", "flag_b": "int"}
DIMENSION_COLTYPES = {"key": "int", "order_day": "date", "segment": "int"}


def _rng(seed: int, name: str) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64([seed, zlib.crc32(name.encode())]))


_LINEITEM = (("quantity", 1, 51, np.int32), ("price_cents", 90_000, 10_500_001, np.int64),
             ("discount_pct", 0, 11, np.int32), ("tax_pct", 0, 9, np.int32),
             ("ship_day", DAY0, DAY0 + NDAYS, np.int32), ("flag_a", 0, 3, np.uint8), ("flag_b", 0, 2, np.uint8))


def _pool() -> ThreadPoolExecutor:
    return ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1))


def lineitem(n: int, seed: int = 1) -> dict[str, np.ndarray]:
    # Each column has its own stream, so drawing them on threads gives the
    # same values as drawing them one after another.
    def draw(spec):
        name, lo, hi, dt = spec
        return name, _rng(seed, name).integers(lo, hi, n, dtype=dt)
    if n < (1 << 20):
        return dict(draw(s) for s in _LINEITEM)
    with _pool() as ex:
        return dict(ex.map(draw, _LINEITEM))


def dimension(n: int, seed: int = 2) -> dict[str, np.ndarray]:
    key = _rng(seed, "key").permutation(np.arange(1, n + 1, dtype=np.int32))
    return {
        "key": key,
        "order_day": _rng(seed, "order_day").integers(DAY0, DAY0 + NDAYS, n, dtype=np.int32),
        "segment": _rng(seed, "segment").integers(0, 25, n, dtype=np.uint8),
    }


def zipf_ranks(n: int, nkeys: int, s: float, rng: np.random.Generator, chunk: int = 1 << 22) -> np.ndarray:
    """n draws of ranks 1..nkeys with P(r) ∝ r^-s (inverse CDF)."""
    w = np.arange(1, nkeys + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    out = np.empty(n, dtype=np.int64)
    # The uniforms are drawn chunk by chunk in order (so the values do not
    # depend on the thread count); the searches run on threads.
    def search(i, u):
        out[i:i + u.shape[0]] = np.searchsorted(cdf, u, side="right") + 1
    with _pool() as ex:
        futs = []
        for i in range(0, n, chunk):
            futs.append(ex.submit(search, i, rng.random(min(chunk, n - i))))
        for f in futs:
            f.result()
    np.minimum(out, nkeys, out=out)
    return out


def fact_fk(n: int, nkeys: int, s: float = 0.8, seed: int = 3) -> dict[str, np.ndarray]:
    t = lineitem(n, seed)
    t["fk"] = zipf_ranks(n, nkeys, s, _rng(seed, "fk")).astype(np.int32)
    return t


def highcard(n: int, nkeys: int = 10_000_000, s: float = 1.1, seed: int = 4) -> dict[str, np.ndarray]:
    return {
        "key": zipf_ranks(n, nkeys, s, _rng(seed, "key")),
        "value": _rng(seed, "value").integers(0, 1001, n, dtype=np.int32),
    }
