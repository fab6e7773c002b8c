"""ctypes mirror of ``include/turbogp_gpu.h`` and the loader of the in-tree library.

The product path is the CUDA library ``libturbogp_b200.so`` next to this file.
There is no CPU fallback: if the library is missing or fails to load, every
entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libturbogp_b200.so"

# --- status codes ----------------------------------------------------------
OK, INVALID_ARG, OOM, UNSUPPORTED, TIMEOUT, DEVICE_ERROR, NOT_FOUND, CAPACITY, PENDING = range(9)

# --- enums -------------------------------------------------------------------
DT_U8, DT_I32, DT_I64, DT_U64, DT_F64 = 1, 2, 3, 4, 5
CT_INT, CT_DATE, CT_FLOAT = 0, 1, 2
CMP_EQ, CMP_NE, CMP_LT, CMP_LE, CMP_GT, CMP_GE, CMP_BETWEEN, CMP_NOT_BETWEEN = range(8)
PN_LEAF, PN_AND, PN_OR, PN_NOT = range(4)
AGG_COUNT_STAR, AGG_COUNT_NONZERO, AGG_SUM, AGG_AVG, AGG_MIN, AGG_MAX = range(6)
SIDE_PROBE, SIDE_BUILD = 0, 1
RESULT_ROW_OVERFLOW = 1

MAX_FACTORS = 4
MAX_AGGS = 8
MAX_GROUP_KEYS = 4
MAX_PRED_NODES = 16


class Variant(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("max_stages", C.c_uint32), ("placement", C.c_uint32),
                ("presum", C.c_uint32), ("dense", C.c_uint32), ("shapes", C.c_uint32), ("payload", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("l2_ahead", C.c_uint32), ("_pad", C.c_uint32)]


class TuneEntry(C.Structure):
    _fields_ = [("variant", Variant), ("ms", C.c_double), ("status", C.c_int32), ("same_result", C.c_uint32),
                ("threads_used", C.c_uint32), ("stages_used", C.c_uint32), ("mode_used", C.c_uint32),
                ("_pad", C.c_uint32)]


class ColumnDesc(C.Structure):
    _fields_ = [("dtype", C.c_uint32), ("coltype", C.c_uint32), ("data", C.c_void_p)]


class CellColumn(C.Structure):
    _fields_ = [("cells", C.c_void_p), ("i32_sidecar", C.c_void_p), ("coltype", C.c_uint32), ("_pad", C.c_uint32)]


class PredNode(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32), ("column", C.c_uint32), ("cmp", C.c_uint32), ("_pad", C.c_uint32),
        ("lit", C.c_uint64), ("lit2", C.c_uint64),
    ]


class Factor(C.Structure):
    _fields_ = [("column", C.c_int32), ("side", C.c_uint32), ("mul", C.c_int64), ("add", C.c_int64)]


class Agg(C.Structure):
    _fields_ = [("func", C.c_uint32), ("nfactors", C.c_uint32), ("f", Factor * MAX_FACTORS)]


class GroupKey(C.Structure):
    _fields_ = [("column", C.c_uint32), ("side", C.c_uint32)]


class Query(C.Structure):
    _fields_ = [
        ("table", C.c_uint64),
        ("pred", C.POINTER(PredNode)), ("npred", C.c_uint32),
        ("ngroup", C.c_uint32), ("group", C.POINTER(GroupKey)),
        ("nagg", C.c_uint32), ("_pad", C.c_uint32), ("aggs", C.POINTER(Agg)),
        ("join", C.c_uint64), ("probe_key_column", C.c_uint32), ("flags", C.c_uint32),
    ]


class AggValue(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_int64), ("count", C.c_uint64), ("as_f64", C.c_double)]

    @property
    def value(self) -> int:
        return (self.hi << 64) | self.lo


class QueryResult(C.Structure):
    _fields_ = [
        ("rows_scanned", C.c_uint64), ("rows_selected", C.c_uint64), ("ngroups", C.c_uint64),
        ("flags", C.c_uint32), ("_pad", C.c_uint32),
    ]


class BatchItem(C.Structure):
    _fields_ = [
        ("query", C.POINTER(Query)), ("keys_out", C.c_void_p), ("vals_out", C.POINTER(AggValue)),
        ("group_cap", C.c_uint64), ("result", QueryResult), ("status", C.c_int32), ("_pad", C.c_uint32),
    ]


class KernelParams(C.Structure):
    _fields_ = [
        ("target_u64", C.c_uint64), ("low_u64", C.c_uint64), ("high_u64", C.c_uint64),
        ("max_distance", C.c_uint32), ("_pad0", C.c_uint32), ("cell_count", C.c_uint64),
        ("target2_u64", C.c_uint64), ("target3_u64", C.c_uint64),
        ("pred1_op", C.c_uint8), ("pred2_op", C.c_uint8), ("pred3_op", C.c_uint8),
        ("predicate_count", C.c_uint8), ("_pad1", C.c_uint32),
    ]


class KeyDomain(C.Structure):
    _fields_ = [("column", C.c_uint32), ("_pad", C.c_uint32), ("min", C.c_int64), ("count", C.c_uint64)]


class KernelResultC(C.Structure):
    _fields_ = [("count", C.c_uint64), ("sum", C.c_double), ("mask", C.c_uint64)]


class KernelInfo(C.Structure):
    _fields_ = [("op", C.c_uint32), ("cpu", C.c_uint32), ("tier", C.c_uint32), ("_pad", C.c_uint32),
                ("name", C.c_char_p)]


# (name, restype, argtypes) for every exported symbol of the header.
PROTOTYPES = [
    ("tgp_status_string", C.c_char_p, [C.c_int]),
    ("tgp_init", C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    ("tgp_shutdown", C.c_int, [C.c_void_p]),
    ("tgp_last_error", C.c_char_p, [C.c_void_p]),
    ("tgp_ctx_stream", C.c_void_p, [C.c_void_p]),
    ("tgp_ctx_sm_count", C.c_int, [C.c_void_p]),
    ("tgp_sync", C.c_int, [C.c_void_p]),
    ("tgp_profile_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("tgp_profile_read", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    ("tgp_kernel_count", C.c_uint32, []),
    ("tgp_kernel_info_at", C.c_int, [C.c_uint32, C.POINTER(KernelInfo)]),
    ("tgp_kernel_execute", C.c_int,
     [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(KernelParams), C.POINTER(KernelResultC)]),
    ("tgp_hash_table_free", C.c_int, [C.c_void_p, C.c_void_p]),
    ("tgp_table_register", C.c_int,
     [C.c_void_p, C.POINTER(ColumnDesc), C.c_uint32, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("tgp_table_register_device", C.c_int,
     [C.c_void_p, C.POINTER(ColumnDesc), C.c_uint32, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("tgp_table_register_cells", C.c_int,
     [C.c_void_p, C.POINTER(CellColumn), C.c_uint32, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("tgp_table_column_dtype", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_uint32)]),
    ("tgp_table_reload", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(ColumnDesc), C.c_uint32]),
    ("tgp_table_drop", C.c_int, [C.c_void_p, C.c_uint64]),
    ("tgp_table_info", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    ("tgp_table_column_stats", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("tgp_filter", C.c_int,
     [C.c_void_p, C.c_uint64, C.POINTER(PredNode), C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64,
      C.POINTER(C.c_uint64)]),
    ("tgp_execute", C.c_int,
     [C.c_void_p, C.POINTER(Query), C.c_void_p, C.POINTER(AggValue), C.c_uint64, C.POINTER(QueryResult)]),
    ("tgp_execute_topn", C.c_int,
     [C.c_void_p, C.POINTER(Query), C.c_uint32, C.c_int, C.c_uint64, C.c_void_p, C.POINTER(AggValue),
      C.POINTER(QueryResult)]),
    ("tgp_join_build_smaller", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(PredNode), C.c_uint32, C.c_uint64, C.c_uint32,
      C.POINTER(PredNode), C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
      C.POINTER(C.c_uint64)]),
    ("tgp_query_footprint", C.c_int, [C.c_void_p, C.POINTER(Query), C.POINTER(C.c_uint64)]),
    ("tgp_strings_register", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("tgp_strings_drop", C.c_int, [C.c_void_p, C.c_uint64]),
    ("tgp_debug_fail_next_scan", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64]),
    ("tgp_like", C.c_int, [C.c_void_p, C.c_uint64, C.c_char_p, C.c_uint32, C.c_int, C.c_void_p,
                           C.POINTER(C.c_uint64)]),
    ("tgp_set_default_variant", C.c_int, [C.c_void_p, C.POINTER(Variant)]),
    ("tgp_get_default_variant", C.c_int, [C.c_void_p, C.POINTER(Variant)]),
    ("tgp_batch_config", C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.c_uint64]),
    ("tgp_tune_class", C.c_int, [C.c_void_p, C.POINTER(Query), C.POINTER(C.c_uint64)]),
    ("tgp_tune_set", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Variant)]),
    ("tgp_tune_get", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Variant), C.POINTER(C.c_int)]),
    ("tgp_tune_count", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    ("tgp_tune_at", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(Variant)]),
    ("tgp_tune_clear", C.c_int, [C.c_void_p]),
    ("tgp_autotune", C.c_int, [C.c_void_p, C.POINTER(Query), C.c_uint32, C.POINTER(TuneEntry), C.c_uint32,
                               C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    ("tgp_count_distinct", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(PredNode), C.c_uint32, C.POINTER(C.c_uint64),
      C.POINTER(C.c_uint32)]),
    ("tgp_hll_estimate", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("tgp_join_build", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(PredNode), C.c_uint32, C.POINTER(C.c_uint64)]),
    ("tgp_join_drop", C.c_int, [C.c_void_p, C.c_uint64]),
    ("tgp_join_probe_pairs", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(PredNode), C.c_uint32, C.c_void_p, C.c_void_p,
      C.c_uint64, C.POINTER(C.c_uint64)]),
    ("tgp_batch_submit", C.c_int, [C.c_void_p, C.POINTER(BatchItem), C.c_uint32, C.POINTER(C.c_uint64)]),
    ("tgp_batch_poll", C.c_int, [C.c_void_p, C.c_uint64, C.c_int]),
    ("tgp_graph_capture", C.c_int, [C.c_void_p, C.POINTER(Query), C.POINTER(C.c_uint64)]),
    ("tgp_graph_launch", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(AggValue), C.c_uint64, C.POINTER(QueryResult)]),
    ("tgp_graph_drop", C.c_int, [C.c_void_p, C.c_uint64]),
    ("tgp_aggregate_noalloc", C.c_int,
     [C.c_int, C.c_void_p, C.POINTER(ColumnDesc), C.c_uint32, C.c_uint64, C.POINTER(PredNode), C.c_uint32,
      C.POINTER(KeyDomain), C.c_uint32, C.POINTER(Agg), C.c_uint32, C.POINTER(AggValue), C.c_uint64,
      C.POINTER(QueryResult), C.c_char_p, C.c_size_t]),
]

NOALLOC_SCRATCH_BYTES = 256 * 1024

_lib: C.CDLL | None = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads the CUDA library (once). Raises if it is absent: there is no fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m turbogp_b200.build` (nvcc, sm_100a). "
            "turbogp_b200 has no CPU fallback.")
    lib = C.CDLL(str(p))
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class TgpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


STATUS_NAMES = {OK: "OK", INVALID_ARG: "INVALID_ARG", OOM: "OOM", UNSUPPORTED: "UNSUPPORTED",
                TIMEOUT: "TIMEOUT", DEVICE_ERROR: "DEVICE_ERROR", NOT_FOUND: "NOT_FOUND",
                CAPACITY: "CAPACITY", PENDING: "PENDING"}
