"""Build recipe of libavism_gpu.so (sm_100a) -- run by __graft_entry__.build().

One nvcc invocation compiles the single translation unit csrc/avism_all.cu plus
the host-side merge (csrc/merge.cpp).  --fmad=false keeps every REAL*4 multiply
and add separately rounded, as the reference's expressions are; division and
square root stay IEEE (no fast-math).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libavism_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "--expt-relaxed-constexpr", "--extended-lambda",
]


def sources():
    return [os.path.join(CSRC, "avism_all.cu"), os.path.join(CSRC, "merge.cpp"), os.path.join(CSRC, "io.cpp")]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "avism_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *NVCC_FLAGS, "-shared", "-o", LIB, *sources(), "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
