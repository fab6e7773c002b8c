"""The C ABI library: it loads on a CPU-only host, exports every symbol the
header declares, and the ctypes mirrors match the C struct layouts."""
import ctypes as C
import re
import subprocess
import sys

import pytest

from conftest import ROOT
from turbogp_b200 import _capi as A

HEADER = ROOT / "include" / "turbogp_gpu.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^TGP_API [^(]*?\b(tgp_\w+)\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    if not A.LIB_PATH.exists():
        import turbogp_b200.build as b
        b.build()
    return A.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    nm = subprocess.run(["nm", "-D", "--defined-only", str(A.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (tgp_\w+)$", nm, flags=re.M))
    assert set(names) <= exported
    assert {p[0] for p in A.PROTOTYPES} == set(names)


def test_status_strings_and_kernel_registry(lib):
    assert lib.tgp_status_string(A.OK) == b"OK"
    assert lib.tgp_status_string(A.CAPACITY) == b"CAPACITY"
    n = lib.tgp_kernel_count()
    names = []
    for i in range(n):
        info = A.KernelInfo()
        assert lib.tgp_kernel_info_at(i, C.byref(info)) == A.OK
        assert info.cpu == 5 and info.tier == 3  # GpuSm100a, Hbm
        names.append(info.name.decode())
    assert n == 7 and len(set(names)) == 7
    assert lib.tgp_kernel_info_at(n, C.byref(A.KernelInfo())) == A.INVALID_ARG


STRUCTS = {
    "tgp_column_desc": (A.ColumnDesc, ["dtype", "coltype", "data"]),
    "tgp_pred_node": (A.PredNode, ["kind", "column", "cmp", "lit", "lit2"]),
    "tgp_factor": (A.Factor, ["column", "side", "mul", "add"]),
    "tgp_agg": (A.Agg, ["func", "nfactors", "f"]),
    "tgp_group_key": (A.GroupKey, ["column", "side"]),
    "tgp_query": (A.Query, ["table", "pred", "npred", "ngroup", "group", "nagg", "aggs", "join",
                            "probe_key_column", "flags"]),
    "tgp_agg_value": (A.AggValue, ["lo", "hi", "count", "as_f64"]),
    "tgp_query_result": (A.QueryResult, ["rows_scanned", "rows_selected", "ngroups", "flags"]),
    "tgp_kernel_params": (A.KernelParams, ["target_u64", "low_u64", "high_u64", "max_distance", "cell_count",
                                           "target2_u64", "target3_u64", "pred1_op", "pred2_op", "pred3_op",
                                           "predicate_count"]),
    "tgp_kernel_result": (A.KernelResultC, ["count", "sum", "mask"]),
    "tgp_kernel_info": (A.KernelInfo, ["op", "cpu", "tier", "name"]),
    "tgp_batch_item": (A.BatchItem, ["query", "keys_out", "vals_out", "group_cap", "result", "status"]),
    "tgp_cell_column": (A.CellColumn, ["cells", "i32_sidecar", "coltype"]),
}


def test_struct_layouts_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for s, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fields:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                              check=True).stdout.splitlines())
    for s, (cls, fields) in STRUCTS.items():
        assert int(out[s]) == C.sizeof(cls), s
        for f in fields:
            assert int(out[f"{s}.{f}"]) == getattr(cls, f).offset, f"{s}.{f}"


def test_no_cpu_fallback_without_a_device(lib):
    # On a host without a usable GPU, opening a context fails loudly.
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert lib.tgp_init(C.byref(h), 0) != A.OK
