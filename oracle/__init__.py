"""TEST INFRASTRUCTURE: loader for the CPU oracle (``oracle.cpp``) and the C++
restatement of the reference's CPU path (``ref_path.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs import this package. The product (``turbogp_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "liboracle.so"
SOURCES = [HERE / "oracle.cpp", HERE / "ref_path.cpp"]
HEADER = HERE.parent / "include" / "turbogp_gpu.h"


def build(force: bool = False) -> Path:
    """Compiles the oracle with g++ (no GPU, no CUDA)."""
    BUILD.mkdir(exist_ok=True)
    srcs = [s for s in SOURCES if s.exists()]
    newest = max(p.stat().st_mtime for p in [*srcs, HEADER])
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC",
               "-o", str(tmp), *map(str, srcs)]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


_cdll = None


def load() -> C.CDLL:
    global _cdll
    if _cdll is None:
        build()
        _cdll = C.CDLL(str(LIB))
    return _cdll


# ---------------------------------------------------------------------------
# Python wrappers (host numpy columns in, engine-shaped results out)
# ---------------------------------------------------------------------------
import numpy as np  # noqa: E402

from turbogp_b200 import _capi as A  # noqa: E402  (POD types only)
from turbogp_b200.engine import (AggResult, FilterOutput, QueryOutput, Schema,  # noqa: E402
                                 decode_groups)


def _descs(columns: dict, schema: Schema):
    arrs = [np.ascontiguousarray(columns[n]) for n in schema.names]
    d = (A.ColumnDesc * max(1, len(arrs)))()
    for i, a in enumerate(arrs):
        d[i].dtype, d[i].coltype, d[i].data = schema.dtypes[i][0], schema.dtypes[i][1], a.ctypes.data
    rows = arrs[0].shape[0] if arrs else 0
    return d, arrs, rows


def _sig(lib):
    lib.orc_filter.argtypes = [C.POINTER(A.ColumnDesc), C.c_uint32, C.c_uint64, C.POINTER(A.PredNode), C.c_uint32,
                               C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]
    lib.orc_execute.argtypes = [C.POINTER(A.ColumnDesc), C.c_uint32, C.c_uint64, C.POINTER(A.Query),
                                C.POINTER(A.ColumnDesc), C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(A.PredNode),
                                C.c_uint32, C.c_void_p, C.POINTER(A.AggValue), C.c_uint64, C.POINTER(A.QueryResult)]
    lib.orc_join_pairs.argtypes = [C.POINTER(A.ColumnDesc), C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(A.PredNode),
                                   C.c_uint32, C.POINTER(A.ColumnDesc), C.c_uint32, C.c_uint64, C.c_uint32,
                                   C.POINTER(A.PredNode), C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64,
                                   C.POINTER(C.c_uint64)]
    lib.orc_xxh3_u64.argtypes = [C.c_uint64]
    lib.orc_xxh3_u64.restype = C.c_uint64
    lib.orc_hll_estimate.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
    lib.orc_hll_estimate.restype = C.c_uint64
    lib.orc_hll_estimate_regs.argtypes = [C.c_void_p]
    lib.orc_hll_estimate_regs.restype = C.c_uint64
    lib.orc_count_distinct.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint32)]
    lib.orc_count_distinct.restype = None
    lib.orc_seq_sum_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
    lib.orc_seq_sum_f64.restype = None
    lib.orc_like.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_char_p, C.c_uint64, C.c_int, C.c_void_p]
    lib.orc_like.restype = C.c_uint64
    lib.orc_kernel_execute.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(A.KernelParams),
                                       C.POINTER(A.KernelResultC)]
    return lib


def _lib():
    lib = load()
    if not getattr(lib, "_typed", False):
        _sig(lib)
        lib._typed = True
    return lib


def filter(columns: dict, coltypes: dict | None, where) -> FilterOutput:
    sc = Schema.of(columns, coltypes)
    d, keep, rows = _descs(columns, sc)
    nodes, n = sc.lower_pred(where)
    bm = np.zeros((rows + 7) // 8, dtype=np.uint8)
    rid = np.zeros(max(1, rows), dtype=np.uint32)
    cnt = C.c_uint64()
    if _lib().orc_filter(d, len(sc.names), rows, nodes, n, bm.ctypes.data if bm.size else None, rid.ctypes.data,
                         C.byref(cnt)) != 0:
        raise ValueError("malformed predicate program")
    c = int(cnt.value)
    return FilterOutput(c, bm, rid[:c].copy())


def aggregate(columns: dict, coltypes: dict | None, aggs, group_by=(), where=None, build=None,
              probe_key: str | None = None) -> QueryOutput:
    """``build`` = (columns, coltypes, key_name, where) of the joined table."""
    sc = Schema.of(columns, coltypes)
    d, keep, rows = _descs(columns, sc)
    bsc = None
    bd, bkeep, brows, bkey, bnodes, nb = None, None, 0, 0, None, 0
    if build is not None:
        bcols, bct, bkey_name, bwhere = build
        bsc = Schema.of(bcols, bct)
        bd, bkeep, brows = _descs(bcols, bsc)
        bkey = bsc.index(bkey_name)
        bnodes, nb = bsc.lower_pred(bwhere)
    q, qkeep = sc.lower_query(aggs, group_by, where, bsc, probe_key)
    q.join = 1 if build is not None else 0
    cap = 1024
    nk, na = len(group_by), len(aggs)
    while True:
        keys = np.zeros(max(1, cap * max(1, nk)), dtype=np.uint64)
        vals = (A.AggValue * max(1, cap * max(1, na)))()
        res = A.QueryResult()
        st = _lib().orc_execute(d, len(sc.names), rows, C.byref(q), bd, len(bsc.names) if bsc else 0, brows, bkey,
                                bnodes, nb, keys.ctypes.data, vals, cap, C.byref(res))
        if st == A.CAPACITY:
            cap = int(res.ngroups)
            continue
        if st != 0:
            raise ValueError("malformed query")
        break
    ks, vs = decode_groups(keys, vals, int(res.ngroups), nk, na)
    return QueryOutput(ks, vs, int(res.rows_scanned), int(res.rows_selected), int(res.flags))


def join_pairs(probe_columns: dict, probe_coltypes, probe_key: str, probe_where, build_columns: dict,
               build_coltypes, build_key: str, build_where):
    psc = Schema.of(probe_columns, probe_coltypes)
    pd, pkeep, prows = _descs(probe_columns, psc)
    bsc = Schema.of(build_columns, build_coltypes)
    bd, bkeep, brows = _descs(build_columns, bsc)
    pn, npn = psc.lower_pred(probe_where)
    bn, nbn = bsc.lower_pred(build_where)
    cnt = C.c_uint64()
    lib = _lib()
    lib.orc_join_pairs(pd, len(psc.names), prows, psc.index(probe_key), pn, npn, bd, len(bsc.names), brows,
                       bsc.index(build_key), bn, nbn, None, None, 0, C.byref(cnt))
    m = int(cnt.value)
    pr = np.zeros(max(1, m), dtype=np.uint32)
    br = np.zeros(max(1, m), dtype=np.uint32)
    lib.orc_join_pairs(pd, len(psc.names), prows, psc.index(probe_key), pn, npn, bd, len(bsc.names), brows,
                       bsc.index(build_key), bn, nbn, pr.ctypes.data, br.ctypes.data, m, C.byref(cnt))
    return pr[:m], br[:m]


def kernel_execute(op: int, cells: np.ndarray, params, probe_cells: np.ndarray | None = None):
    """Scalar kernel-table semantics; for HashProbe pass the build keys as
    ``cells`` and the probe keys as ``probe_cells``. Returns (count, sum, mask)."""
    a = np.ascontiguousarray(cells, dtype=np.uint64)
    b = np.ascontiguousarray(probe_cells if probe_cells is not None else np.zeros(0), dtype=np.uint64)
    p = params.to_c() if hasattr(params, "to_c") else params
    p.cell_count = a.shape[0]
    r = A.KernelResultC()
    if _lib().orc_kernel_execute(op, a.ctypes.data if a.size else None, b.ctypes.data if b.size else None,
                                 b.shape[0], C.byref(p), C.byref(r)) != 0:
        raise ValueError("operator without an oracle")
    return int(r.count), float(r.sum), int(r.mask)


def xxh3_u64(v: int) -> int:
    """xxh3_64 of the 8 little-endian bytes of a cell (the oracle's restatement)."""
    return int(_lib().orc_xxh3_u64(v & 0xFFFFFFFFFFFFFFFF))


def hll_estimate(cells: np.ndarray, sel_bitmap: np.ndarray | None = None) -> int:
    """The reference's HyperLogLog estimate over the (selected) u64 cells."""
    c = np.ascontiguousarray(cells).view(np.uint64)
    return int(_lib().orc_hll_estimate(c.ctypes.data if c.size else None, c.shape[0],
                                       sel_bitmap.ctypes.data if sel_bitmap is not None else None))


def count_distinct(cells: np.ndarray, sel_bitmap: np.ndarray | None = None) -> tuple[int, str]:
    """COUNT(DISTINCT) of u64 cells as the reference evaluates it: (count,
    'exact' | 'hll')."""
    c = np.ascontiguousarray(cells).view(np.uint64)
    cnt, method = C.c_uint64(), C.c_uint32()
    _lib().orc_count_distinct(c.ctypes.data if c.size else None, c.shape[0],
                              sel_bitmap.ctypes.data if sel_bitmap is not None else None, C.byref(cnt),
                              C.byref(method))
    return int(cnt.value), ("hll" if method.value else "exact")


def flat_strings(values) -> tuple[np.ndarray, np.ndarray]:
    """(bytes, offsets) of a list of str / bytes: the flat column layout."""
    bs = [v.encode("utf-8") if isinstance(v, str) else bytes(v) for v in values]
    offs = np.zeros(len(bs) + 1, dtype=np.uint64)
    if bs:
        offs[1:] = np.cumsum([len(b) for b in bs], dtype=np.uint64)
    return np.frombuffer(b"".join(bs), dtype=np.uint8).copy(), offs


def like(values, pattern, negated: bool = False) -> FilterOutput:
    """``col [NOT] LIKE pattern`` as the reference evaluates it, over a list
    of strings (or a (bytes, offsets) pair): (count, LSB-first bitmap)."""
    data, offs = values if isinstance(values, tuple) else flat_strings(values)
    p = pattern.encode("utf-8") if isinstance(pattern, str) else bytes(pattern)
    n = offs.shape[0] - 1
    bm = np.zeros(max(1, (n + 7) // 8), dtype=np.uint8)
    cnt = _lib().orc_like(data.ctypes.data if data.size else None, offs.ctypes.data, n, p, len(p),
                          1 if negated else 0, bm.ctypes.data)
    return FilterOutput(int(cnt), bm[:(n + 7) // 8])
