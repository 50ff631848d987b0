"""Build recipe of libavism_gpu.so (sm_100a) -- run by __graft_entry__.build().

Each CUDA source under csrc/ is its own translation unit (no relocatable
device code: kernels that several units launch live in headers); the units
compile in parallel into csrc/../_build/ and link with the host-side merge
(csrc/merge.cpp) and the file formats (csrc/io.cpp) into one shared library.
--fmad=false keeps every REAL*4 multiply and add separately rounded, as the
reference's expressions are; division and square root stay IEEE (no fast-math).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libavism_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "--expt-relaxed-constexpr", "--extended-lambda",
]


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    return [os.path.join(CSRC, f) for f in cu] + [os.path.join(CSRC, "merge.cpp"), os.path.join(CSRC, "io.cpp")]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "avism_gpu.h"))
    return hs


def _obj(src):
    return os.path.join(OBJ, os.path.basename(src) + ".o")


def _stale_obj(src, hmax) -> bool:
    o = _obj(src)
    return not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(src), hmax)


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + _headers()
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    cmd = [NVCC, *NVCC_FLAGS, "-c", src, "-o", _obj(src)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    hmax = max(os.path.getmtime(h) for h in _headers())
    todo = [s for s in sources() if force or _stale_obj(s, hmax)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        for src, rc, out in ex.map(lambda s: _compile(s, verbose), todo):
            if rc != 0:
                raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{out}")
    cmd = [NVCC, *NVCC_FLAGS, "-shared", "-o", LIB, *(_obj(s) for s in sources()), "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
