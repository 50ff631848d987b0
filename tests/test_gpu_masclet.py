"""GPU parity for MASCLET input (FLAG_DATA = 0) at levels 0 and -1: the level's
U1CO / DIVERCO and whole catalogue through the C-ABI against the oracle, bit
for bit, for the FLAG_DENS / FLAG_DIV choices (src/avism.f90:1366-1405,
1633-1650); a snapshot read from its three files; levels above 0 refused."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O

import masclet_case as mc

pytestmark = pytest.mark.gpu

CASES = [(0, 0, 0), (1, 1, 0), (2, 2, 0), (0, -1, 0), (0, 0, -1), (2, 2, -1), (2, 1, -1)]


@pytest.fixture(scope="module")
def snap():
    return mc.snapshot()


def params(s, fd, fv, lev, periodic=1):
    return Params(nx=s["ng"] >> (-lev), periodic=periodic, lado0=s["box"], level=lev, levmin=lev, flag_dens=fd,
                  flag_div=fv)


@pytest.mark.parametrize("fd,fv,lev", CASES)
def test_fields_and_level_exact(gpu, snap, fd, fv, lev):
    p = params(snap, fd, fv, lev)
    needs_dm = fd <= 1 or fv in (0, 1)
    parts = mc.particles(snap) if needs_dm else None
    u1o, dvo, mdo = O.masclet_fields(p, snap["ng"], mc.gas(snap), parts)
    u1g, dvg, mdg = gpu.masclet_fields(p, snap["ng"], mc.gas(snap), parts)
    assert np.array_equal(u1o, u1g) and np.array_equal(dvo, dvg) and mdo == mdg
    o = O.run_level_masclet(p, snap["ng"], mc.gas(snap), parts)
    g = gpu.run_level_masclet(p, snap["ng"], mc.gas(snap), parts, capacity=200000)
    assert g["nvoid"] == o["vf"]["nvoid"]
    if lev == 0:
        assert g["nvoid"] > 0                    # (at 16^3 the mock's voids fall below NCELL_MIN)
    for k in g["cubes"]:
        assert np.array_equal(g["cubes"][k], o["vf"]["cubes"][k]), k
    for k in ("indice", "uvoid", "ncellv", "volnew", "req", "gxc", "gyc", "gzc", "eps", "ip", "umean", "mtot"):
        assert np.array_equal(g["cat"][k], o["cat"][k]), k


def test_nonperiodic_and_tsc(gpu, snap):
    p = params(snap, 0, 0, 0, periodic=0)
    p.flag_vel_interp = 0
    p.flag_dens_interp = 0
    parts = mc.particles(snap)
    o = O.run_level_masclet(p, snap["ng"], mc.gas(snap), parts)
    g = gpu.run_level_masclet(p, snap["ng"], mc.gas(snap), parts, capacity=200000)
    assert g["nvoid"] == o["vf"]["nvoid"]
    for k in ("indice", "uvoid", "ncellv", "volnew", "umean", "mtot"):
        assert np.array_equal(g["cat"][k], o["cat"][k]), k


def test_from_files(gpu, snap, tmp_path):
    from avism_b200.avism import read_masclet_files
    r = read_masclet_files(*mc.write_files(snap, str(tmp_path)), snap["ng"])
    p = params(snap, 0, 0, 0)
    gas = tuple(r["gas"][k] for k in ("u1g", "u2g", "u3g", "u4g"))
    a = gpu.run_level_masclet(p, snap["ng"], gas, r["parts"], capacity=200000)
    b = gpu.run_level_masclet(p, snap["ng"], mc.gas(snap), mc.particles(snap), capacity=200000)
    for k in a["cat"]:
        assert np.array_equal(np.asarray(a["cat"][k]), np.asarray(b["cat"][k])), k


def test_level_above_zero_is_unsupported(gpu, snap):
    from avism_b200.avism import AvismError
    p = Params(nx=2 * snap["ng"], periodic=1, lado0=snap["box"], level=1)
    with pytest.raises(AvismError) as e:
        gpu.masclet_fields(p, snap["ng"], mc.gas(snap), mc.particles(snap))
    assert "not implemented" in str(e.value)
