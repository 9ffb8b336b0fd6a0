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
                                      "lg_serve.cpp")]
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
    if not force and up_to_date():
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, "-ccbin", "g++", "-o", str(tmp), *map(str, SOURCES)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
