"""Build step for liblgpu.so (sm_100a) into ligerito-rust_b200/_build/.

Run directly (``python ligerito-rust_b200/build_lib.py``) or through
``__graft_entry__.build()``.  Rebuilds only when a source is newer than the
library.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
OUT = PKG / "_build" / "liblgpu.so"
SOURCES = [PKG / "csrc" / f for f in ("lg_api.cu", "lg_kernels.cu", "lg_fs.cu", "lg_host.cpp", "lg_noalloc.cu",
                                      "lg_serve.cpp", "lg_peaks.cu")]
DEPS = SOURCES + [PKG / "csrc" / f for f in ("lg_device.cuh", "lg_fs.cuh", "lg_kernels.h", "lg_host.h")] + [
    ROOT / "include" / "ligerito_b200.h"
]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-pthread", "-shared", "-cudart", "static",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile each source to an object in parallel (a source is recompiled
    when it or any header is newer than its object), then link the shared
    library."""
    if not force and up_to_date():
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    OUT.parent.mkdir(parents=True, exist_ok=True)
    headers = [p for p in DEPS if p not in SOURCES]
    newest_header = max(p.stat().st_mtime for p in headers)
    compile_flags = [f for f in NVCC_FLAGS if f not in ("-shared", "-cudart", "static")]

    def obj(src: pathlib.Path) -> pathlib.Path:
        o = OUT.parent / (src.name + ".o")
        if force or not o.exists() or o.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            cmd = [nvcc(), *compile_flags, "-ccbin", "g++", "-c", "-o", str(o) + ".tmp", str(src)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            os.replace(str(o) + ".tmp", o)
        return o

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(obj, SOURCES))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", "g++",
           "-Xcompiler", "-pthread", "-o", str(tmp), *map(str, objs)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
