"""The C-ABI from C: include/avism_gpu.h compiles as strict C99 (no C++ types in
the boundary), every declared entry point links against libavism_gpu.so, and
the host-only geometry call agrees with the oracle when called from C.  Runs
without a GPU (the context call must fail cleanly there)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from avism_b200 import _lib

from test_lib import declared_functions

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_program(names):
    refs = ",\n    ".join(f"(void (*)(void))(uintptr_t){n}" for n in names)
    return f"""
#include <stdint.h>
#include <stdio.h>
#include "avism_gpu.h"

/* every entry point the header declares, by address: all must link */
static void (*const entry_points[])(void) = {{
    {refs}
}};

int main(int argc, char **argv) {{
    avism_params p = {{0}};
    avism_grid g;
    float radx[4096];
    int st;
    (void)argc;
    p.nx = 64; p.periodic = 1; p.lado0 = 100.0f;
    if (argv[1][0] == 'n') {{ p.nx = 48; p.periodic = 0; p.lado0 = 147.5f; }}
    st = avism_gpu_grid_setup(&p, &g, radx);
    printf("%d %zu\\n", st, sizeof entry_points / sizeof entry_points[0]);
    printf("%d %d %d %d %d %d %d\\n", g.nx, g.nplus, g.low1, g.low2, g.ne, g.rad_lo, g.rad_hi);
    for (int i = 0; i <= g.rad_hi - g.rad_lo; i++) printf("%a\\n", (double)radx[i]);
    {{
        avism_gpu_ctx *ctx = NULL;
        st = avism_gpu_create(&ctx, 0);
        printf("create %d %d\\n", st, ctx == NULL);
        if (ctx) avism_gpu_destroy(ctx);
    }}
    return 0;
}}
"""


@pytest.fixture(scope="module")
def c_binary(tmp_path_factory):
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    lib = _lib.load()
    assert lib is not None
    d = tmp_path_factory.mktemp("cabi")
    src = d / "abi.c"
    src.write_text(_c_program(declared_functions()))
    exe = d / "abi"
    libdir = os.path.join(ROOT, "avism_b200")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                        "-I", os.path.join(ROOT, "include"), str(src), "-L", libdir, "-lavism_gpu",
                        f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


@pytest.mark.parametrize("case", ["periodic", "nonperiodic"])
def test_c_caller_geometry_matches_oracle(c_binary, case):
    from avism_b200._abi import Params
    from oracle import oracle as O
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([c_binary, case], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    st, nent = map(int, lines[0].split())
    assert st == 0 and nent == len(declared_functions())
    nx, nplus, low1, low2, ne, rlo, rhi = map(int, lines[1].split())
    p = Params(nx=48, periodic=0, lado0=147.5) if case == "nonperiodic" else Params(nx=64, periodic=1, lado0=100.0)
    g, radx = O.grid_setup(p)
    assert (nx, nplus, low1, low2, ne, rlo, rhi) == (g.nx, g.nplus, g.low1, g.low2, g.ne, g.rad_lo, g.rad_hi)
    rad_c = np.array([float.fromhex(s) for s in lines[2:2 + (rhi - rlo + 1)]], np.float32)
    assert np.array_equal(rad_c, np.asarray(radx, np.float32))
    # no GPU visible: the context call reports AVISM_ERR_NO_DEVICE and hands back no context
    assert lines[-1] == "create 7 1"
