"""Build libcardiotrust_cuda.so (sm_100a) in-tree with nvcc.

Every translation unit is compiled with -fmad=false: the kernels write
fmaf() exactly where the reference crate calls mul_add and keep every other
product and sum separately rounded. Host code is compiled with
-ffp-contract=off for the same reason.
"""

from __future__ import annotations

import os
import pathlib
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libcardiotrust_cuda.so"
BUILD_DIR = PKG / "_build"

SOURCES = ["ct_api.cu", "ct_propagate.cu", "ct_measure.cu", "ct_derive.cu", "ct_update.cu", "ct_umma.cu", "ct_adjoint.cu", "ct_plain.cu",
           "ct_post.cu", "ct_model.cu", "ct_slice.cu"]
HEADERS = ["ct_internal.cuh", "ct_sync.cuh", "ct_tcgen05.cuh"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-fmad=false",
    "-Xcompiler",
    "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas",
    "-O3",
]


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    BUILD_DIR.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "cardiotrust_cuda.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD_DIR / (src[:-3] + ".o")
        if force or _stale(o, [s, *headers]):
            cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.check_call(cmd)
        objs.append(o)
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(f".{os.getpid()}.tmp")
        cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
