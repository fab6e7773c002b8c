"""Builds the in-tree CUDA library ``turbogp_b200/libturbogp_b200.so`` for sm_100a.

Every translation unit under ``csrc/`` is compiled with nvcc for
``arch=compute_100a,code=sm_100a`` and linked into one shared library with the
CUDA runtime linked statically, so the library loads on any box with a
recent driver without depending on the process's LD_LIBRARY_PATH.
Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build" / "turbogp_b200"
LIB = PKG / "libturbogp_b200.so"
SOURCES = ["scan_engine.cu", "aux_kernels.cu", "groupby_direct.cu", "capi.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--diag-suppress=128,177", f"-I{ROOT / 'include'}", f"-I{CSRC}",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build turbogp_b200")
    return exe


def _headers() -> list[Path]:
    return list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "turbogp_gpu.h"]


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *_headers()])


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    jobs = []
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD / (Path(name).stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
            for f in [ex.submit(_compile, s, o, verbose) for s, o in jobs]:
                f.result()
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
