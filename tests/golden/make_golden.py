"""Writes the golden fixtures of tests/test_golden.py from the CPU oracle.

The reference (Fortran, no compiler in this image) cannot produce outputs
here, so these fixtures freeze the oracle's results on small seeded inputs:
a change in the oracle or in the CUDA path that alters any of them shows up
as a test failure.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from avism_b200 import synth  # noqa: E402
from avism_b200._abi import Params  # noqa: E402
from oracle import oracle as O  # noqa: E402


def level_case():
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=64.0, nsph=3, rmin=5.0, rmax=9.0, seed=7))
    out = {}
    for per in (1, 0):
        p = Params(nx=32, periodic=per, lado0=64.0)
        r = O.run_level(p, parts)
        out[f"p{per}_nvoid"] = np.int32(r["vf"]["nvoid"])
        out[f"p{per}_meandens"] = np.float32(r["meandens"])
        for k, v in r["vf"]["cubes"].items():
            out[f"p{per}_cube_{k}"] = np.asarray(v)
        for k in ("indice", "uvoid", "ncellv", "volnew", "req", "gxc", "gyc", "gzc", "xc", "yc", "zc"):
            out[f"p{per}_cat_{k}"] = np.asarray(r["cat"][k])
        out[f"p{per}_nvoidt"] = np.int32(r["cat"]["nvoidt"])
        out[f"p{per}_u_mass"] = np.asarray(r["grid"]["u_mass"])
    return out


def knn_case():
    rng = np.random.default_rng(20261203)
    x, y, z = (rng.uniform(-25, 25, 3000).astype(np.float32) for _ in range(3))
    qx, qy, qz = (rng.uniform(-25, 25, 500).astype(np.float32) for _ in range(3))
    out = {"x": x, "y": y, "z": z, "qx": qx, "qy": qy, "qz": qz}
    for L in (50.0, 0.0):
        i, d = O.knn(x, y, z, qx, qy, qz, 8, L)
        tag = "per" if L > 0 else "open"
        out[f"{tag}_idx"] = np.asarray(i)
        out[f"{tag}_dist"] = np.asarray(d)
    return out


def indexx_case():
    rng = np.random.default_rng(5)
    a = rng.integers(0, 40, 2000).astype(np.float32)          # many equal keys
    return {"arr": a, "indx": np.asarray(O.indexx(a))}


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "level_mock32.npz"), **level_case())
    np.savez_compressed(os.path.join(HERE, "knn_3000.npz"), **knn_case())
    np.savez_compressed(os.path.join(HERE, "indexx_ties.npz"), **indexx_case())
    print("written")
