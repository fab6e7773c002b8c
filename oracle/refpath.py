"""TEST / BASELINE INFRASTRUCTURE: Python driver of ``ref_path.cpp`` (the C++
restatement of the reference's CPU execution of the benchmark queries)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import load


class RefLeaf(C.Structure):
    _fields_ = [("col", C.c_uint32), ("op", C.c_uint32), ("sgn", C.c_uint32), ("_pad", C.c_uint32),
                ("lit", C.c_uint64), ("lit2", C.c_uint64)]


_OPS = {0: 0, 1: 1, 2: 2, 3: 3, 4: 4, 5: 5, 6: 6}  # tgp_cmp -> ref op (BETWEEN = 6)
COLTYPES = {"ship_day": "date", "discount_pct": "int", "quantity": "int", "price_cents": "int"}


def to_cells(a: np.ndarray) -> np.ndarray:
    """The reference's storage: one u64 cell per value (sign-extended)."""
    return a.astype(np.int64).view(np.uint64) if a.dtype != np.uint64 else a


def selective_scan_sum(cols: dict, tpl, threads: int | None = None) -> dict:
    """Runs the conjunction + SUM(a*b) + COUNT template the reference's way.

    ``cols`` holds native-width numpy columns; they are widened to u64 cells
    outside the timed region (that is the reference's table layout)."""
    lib = load()
    fn = lib.ref_scan_sum_mul
    fn.restype = C.c_double
    fn.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.POINTER(RefLeaf), C.c_uint32, C.c_uint32, C.c_uint32,
                   C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    names = list(cols)
    cells = [np.ascontiguousarray(to_cells(cols[n])) for n in names]
    ptrs = (C.c_void_p * len(cells))(*[c.ctypes.data for c in cells])
    leaves = []
    for op in tpl.where.ops:
        if op[0] == "and":
            continue
        if op[0] != "leaf":
            raise ValueError("the scan baseline takes a conjunction of leaves")
        _, name, cmp, v, v2 = op
        L = RefLeaf()
        L.col, L.op = names.index(name), _OPS[cmp]
        L.sgn = 1 if COLTYPES.get(name, "int") == "int" else 0
        L.lit, L.lit2 = int(v) & 0xFFFFFFFFFFFFFFFF, int(v2) & 0xFFFFFFFFFFFFFFFF
        leaves.append(L)
    arr = (RefLeaf * len(leaves))(*leaves)
    (f_a, f_b) = tpl.aggs[0].term.factors
    s, c = C.c_double(), C.c_uint64()
    sec = fn(ptrs, cells[0].shape[0], arr, len(leaves), names.index(f_a.column), names.index(f_b.column),
             C.byref(s), C.byref(c))
    return {"seconds": sec, "sum": s.value, "count": int(c.value), "threads": 1}
