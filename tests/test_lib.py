"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

from avism_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(avism_(?:gpu|io)_\w+)\s*\(", text))
    return sorted(names)


def test_library_builds_and_loads():
    from avism_b200 import build
    build.build()
    lib = _lib.load()
    assert isinstance(lib, ctypes.CDLL)


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.avism_gpu_create(ctypes.byref(h), 0) == 7      # AVISM_ERR_NO_DEVICE
    assert not h.value


def test_grid_setup_matches_oracle_on_host():
    # the geometry entry point is host-only; it must agree with the oracle bit for bit
    import numpy as np
    from avism_b200._abi import Params
    from avism_b200.avism import grid_setup
    from oracle import oracle as O
    for nx, L, per in [(64, 100.0, 1), (256, 250.0, 1), (48, 147.5, 0)]:
        p = Params(nx=nx, lado0=L, periodic=per)
        g1, r1 = grid_setup(p)
        g2, r2 = O.grid_setup(p)
        assert np.array_equal(r1, r2)
        assert bytes(g1) == bytes(g2)
