"""Golden fixtures (tests/golden/, written by tests/golden/make_golden.py from
the oracle): the oracle must reproduce them (CPU) and the CUDA path must match
them bit for bit through the C-ABI (GPU)."""
import os

import numpy as np
import pytest

from avism_b200 import synth
from avism_b200._abi import Params
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def _mock():
    return synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=64.0, nsph=3, rmin=5.0, rmax=9.0, seed=7))


def _check_level(gold, per, r_nvoid, cubes, cat, nvoidt):
    assert r_nvoid == int(gold[f"p{per}_nvoid"])
    for k, v in cubes.items():
        assert np.array_equal(np.asarray(v), gold[f"p{per}_cube_{k}"]), k
    for k in ("indice", "uvoid", "ncellv", "volnew", "req", "gxc", "gyc", "gzc", "xc", "yc", "zc"):
        assert np.array_equal(np.asarray(cat[k]), gold[f"p{per}_cat_{k}"]), k
    assert nvoidt == int(gold[f"p{per}_nvoidt"])


def test_oracle_reproduces_level_fixture():
    gold = _load("level_mock32.npz")
    parts = _mock()
    for per in (1, 0):
        r = O.run_level(Params(nx=32, periodic=per, lado0=64.0), parts)
        _check_level(gold, per, r["vf"]["nvoid"], r["vf"]["cubes"], r["cat"], r["cat"]["nvoidt"])
        assert np.array_equal(r["grid"]["u_mass"], gold[f"p{per}_u_mass"])


def test_oracle_reproduces_masclet_fixture():
    """The MASCLET snapshot's level 0 and its level 1 from the patches inside
    the level-0 voids (tests/golden/masclet32.npz)."""
    import sys
    sys.path.insert(0, GOLD)
    import make_golden as mg
    gold = _load("masclet32.npz")
    got = mg.masclet_case()
    assert set(got) == set(gold)
    for k, v in got.items():
        assert np.array_equal(np.asarray(v), gold[k]), k


def test_oracle_reproduces_knn_and_indexx_fixtures():
    g = _load("knn_3000.npz")
    for L, tag in ((50.0, "per"), (0.0, "open")):
        i, d = O.knn(g["x"], g["y"], g["z"], g["qx"], g["qy"], g["qz"], 8, L)
        assert np.array_equal(i, g[f"{tag}_idx"]) and np.array_equal(d, g[f"{tag}_dist"])
    t = _load("indexx_ties.npz")
    assert np.array_equal(O.indexx(t["arr"]), t["indx"])


@pytest.mark.gpu
def test_gpu_matches_level_fixture(gpu):
    gold = _load("level_mock32.npz")
    parts = _mock()
    for per in (1, 0):
        p = Params(nx=32, periodic=per, lado0=64.0)
        r = gpu.run_level(p, parts, capacity=20000)
        _check_level(gold, per, r["nvoid"], r["cubes"], r["cat"], r["cat"]["nvoidt"])
        assert r["meandens"] == gold[f"p{per}_meandens"]
        g2 = gpu.particles_to_grid(p, parts)
        assert np.array_equal(g2["u_mass"], gold[f"p{per}_u_mass"])


@pytest.mark.gpu
def test_gpu_matches_knn_and_indexx_fixtures(gpu):
    g = _load("knn_3000.npz")
    for L, tag in ((50.0, "per"), (0.0, "open")):
        i, d = gpu.knn_search(g["x"], g["y"], g["z"], g["qx"], g["qy"], g["qz"], 8, L)
        assert np.array_equal(i, g[f"{tag}_idx"]) and np.array_equal(d, g[f"{tag}_dist"])
    t = _load("indexx_ties.npz")
    assert np.array_equal(gpu.indexx(t["arr"]), t["indx"])
