"""The committed Rust binding (integration/rust/src/kernel/gpu_ffi.rs) against
the C header it binds, on the CPU: every #[repr(C)] struct has the header
struct's field order, offsets and size (the header compiled with gcc, the
Rust layout computed with the C layout rules #[repr(C)] follows), every
constant has the header's value, and every TGP_API function is declared with
the same number of arguments. (No Rust toolchain exists in this image, so
this is what checks the binding.)"""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
FFI = ROOT / "integration" / "rust" / "src" / "kernel" / "gpu_ffi.rs"
HEADER = ROOT / "include" / "turbogp_gpu.h"

PRIM = {"u8": (1, 1), "i8": (1, 1), "u16": (2, 2), "i16": (2, 2), "u32": (4, 4), "i32": (4, 4), "c_int": (4, 4),
        "f32": (4, 4), "u64": (8, 8), "i64": (8, 8), "f64": (8, 8), "usize": (8, 8), "isize": (8, 8)}


def rust_structs(text):
    structs = {}
    for m in re.finditer(r"#\[repr\(C\)\]\s*(?:#\[derive\([^)]*\)\]\s*)?pub struct (\w+) \{(.*?)\n\}", text, re.S):
        fields = re.findall(r"^\s*(?:pub )?(\w+): ([^,\n]+),", m.group(2), re.M)
        structs[m.group(1)] = [(n, t.strip()) for n, t in fields]
    return structs


def rust_consts(text):
    return {n: v for n, v in re.findall(r"^pub const (\w+): \w+ = ([^;]+);", text, re.M)}


def layout(structs, name):
    """(size, align, {field: offset}) of a #[repr(C)] struct."""
    off, align, offs = 0, 1, {}
    for fname, ftype in structs[name]:
        sz, al = type_layout(structs, ftype)
        off = (off + al - 1) // al * al
        offs[fname] = off
        off += sz
        align = max(align, al)
    return (off + align - 1) // align * align, align, offs


def type_layout(structs, t):
    t = t.strip()
    if t.startswith("*"):
        return 8, 8
    m = re.fullmatch(r"\[(.+); (\w+)\]", t)
    if m:
        sz, al = type_layout(structs, m.group(1))
        n = int(m.group(2)) if m.group(2).isdigit() else {"TGP_MAX_FACTORS": 4}[m.group(2)]
        return sz * n, al
    if t in PRIM:
        return PRIM[t]
    if t in structs:
        sz, al, _ = layout(structs, t)
        return sz, al
    raise ValueError(f"unknown Rust type {t}")


@pytest.fixture(scope="module")
def parsed():
    text = FFI.read_text()
    return text, rust_structs(text), rust_consts(text)


@pytest.fixture(scope="module")
def c_layout(parsed, tmp_path_factory):
    """sizeof / offsetof of every header struct the binding mirrors, and the
    value of every constant it declares, as gcc sees the header."""
    _, structs, consts = parsed
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for s, fields in structs.items():
        if s == "tgp_ctx":
            continue
        lines.append(f'printf("S {s} %zu\\n", sizeof({s}));')
        for f, _ in fields:
            lines.append(f'printf("F {s} {f} %zu\\n", offsetof({s}, {f}));')
    for c in consts:
        lines.append(f'printf("C {c} %lld\\n", (long long)({c}));')
    lines.append("return 0; }")
    d = tmp_path_factory.mktemp("rustshim")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    sizes, offs, vals = {}, {}, {}
    for ln in out.splitlines():
        p = ln.split()
        if p[0] == "S":
            sizes[p[1]] = int(p[2])
        elif p[0] == "F":
            offs[(p[1], p[2])] = int(p[3])
        else:
            vals[p[1]] = int(p[2])
    return sizes, offs, vals


def test_every_header_struct_has_a_twin(parsed):
    _, structs, _ = parsed
    header_structs = set(re.findall(r"typedef struct (tgp_\w+) \{", HEADER.read_text()))
    assert header_structs <= set(structs), sorted(header_structs - set(structs))


def test_struct_layouts_match_the_header(parsed, c_layout):
    _, structs, _ = parsed
    sizes, offs, _ = c_layout
    for s in structs:
        if s == "tgp_ctx":
            continue
        size, _, fo = layout(structs, s)
        assert size == sizes[s], (s, size, sizes[s])
        for f, o in fo.items():
            assert o == offs[(s, f)], (s, f, o, offs[(s, f)])


def test_constants_match_the_header(parsed, c_layout):
    _, _, consts = parsed
    _, _, vals = c_layout
    for name, v in consts.items():
        expr = v.replace("_", "") if re.fullmatch(r"[\d_]+", v) else v
        rust_val = eval(expr, {"__builtins__": {}})   # integer literals and products only
        assert rust_val == vals[name], (name, rust_val, vals[name])


def test_every_function_is_declared_with_its_arity(parsed):
    text, _, _ = parsed
    header = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    c_fns = {}
    for m in re.finditer(r"^TGP_API [^(]*?\b(tgp_\w+)\((.*?)\);", header, re.M | re.S):
        args = m.group(2).strip()
        c_fns[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    block = text[text.index('extern "C" {'):]
    r_fns = {}
    for m in re.finditer(r"pub fn (tgp_\w+)\((.*?)\)", block, re.S):
        args = [a for a in m.group(2).split(",") if a.strip()]
        r_fns[m.group(1)] = len(args)
    assert set(c_fns) == set(r_fns), (sorted(set(c_fns) - set(r_fns)), sorted(set(r_fns) - set(c_fns)))
    for f, n in c_fns.items():
        assert r_fns[f] == n, (f, n, r_fns[f])


def test_build_script_compiles_the_cuda_sources_for_sm100a():
    """build.rs compiles every CUDA translation unit the Python build compiles,
    with the same architecture flag, into the library it links."""
    from turbogp_b200 import build as b
    text = (ROOT / "integration" / "rust" / "build.rs").read_text()
    for src in b.SOURCES:
        assert f'"{src}"' in text
    assert '"arch=compute_100a,code=sm_100a"' in text
    assert "cargo:rustc-link-lib=dylib=turbogp_b200" in text
