"""A C program shaped like the Fortran driver (tests/c_driver.c: host arrays it
owns, the avism_cubes / avism_voids descriptors, one avism_gpu_run_level call)
gets the same catalogue as the ctypes binding, bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from avism_b200._abi import CUBE_FLT, CUBE_INT, VOID_FLT, VOID_INT, Params

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def c_driver(tmp_path_factory):
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("cdriver")
    exe = d / "c_driver"
    libdir = os.path.join(ROOT, "avism_b200")
    r = subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-pedantic",
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c_driver.c"),
                        "-L", libdir, "-lavism_gpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return d, str(exe)


def test_c_driver_matches_ctypes_binding(gpu, mock1, c_driver):
    d, exe = c_driver
    p = Params(nx=64, periodic=1, lado0=100.0, nvoid_max=100000)
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")
    n = len(mock1["x"])
    with open(d / "in.bin", "wb") as f:
        f.write(bytes(p.to_c()))
        f.write(np.int64(n).tobytes())
        for k in keys:
            f.write(np.ascontiguousarray(mock1[k], np.float32).tobytes())
    r = subprocess.run([exe, str(d / "in.bin"), str(d / "out.bin")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    buf = (d / "out.bin").read_bytes()
    nvoid = int(np.frombuffer(buf, np.int32, 1, 0)[0])
    meandens = float(np.frombuffer(buf, np.float32, 1, 4)[0])
    nvoid2, nvoidt = (int(v) for v in np.frombuffer(buf, np.int32, 2, 8))
    volt = float(np.frombuffer(buf, np.float64, 1, 16)[0])
    off = 24
    cols = {}
    for names, dt in ((CUBE_INT, np.int32), (CUBE_FLT, np.float32), (VOID_INT, np.int32), (VOID_FLT, np.float32)):
        for k in names:
            cols[k] = np.frombuffer(buf, dt, nvoid, off)
            off += 4 * nvoid
    assert off == len(buf)
    ref = gpu.run_level(p, mock1, capacity=p.nvoid_max)
    assert nvoid == ref["nvoid"] > 0
    assert meandens == ref["meandens"]
    assert (nvoid2, nvoidt) == (ref["cat"]["nvoid2"], ref["cat"]["nvoidt"])
    assert volt == ref["cat"]["volt_clean"]
    for k in CUBE_INT + CUBE_FLT:
        assert np.array_equal(cols[k], ref["cubes"][k]), k
    for k in VOID_INT + VOID_FLT:
        assert np.array_equal(cols[k], np.asarray(ref["cat"][k])), k
