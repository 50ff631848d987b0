"""GPU parity of grid input (FLAG_DATA = 2, src/avism.f90:1316-1362): the
level's fields from READ_BINARY_GRID's grids at level 0 and, through SMOOTH_2,
below it, and the whole level's catalogue, bit for bit against the oracle."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O
from test_grid_input import grid_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lev,periodic", [(0, 1), (-1, 1), (-2, 0), (-1, 0)])
def test_grid_level_exact(gpu, lev, periodic):
    u1, vs = grid_case()
    nx = 64 >> -lev
    p = Params(nx=nx, periodic=periodic, lado0=100.0, level=lev, levmin=lev, rmin=2.0)
    o = O.grid_fields(p, 64, u1, *vs)
    g = gpu.grid_fields(p, 64, u1, *vs)
    assert np.array_equal(o[0], g[0]) and np.array_equal(o[1], g[1]) and o[2] == g[2]
    ro = O.run_level_grid(p, 64, u1, *vs)
    rg = gpu.run_level_grid(p, 64, u1, *vs, capacity=200000, want_marca=True)
    assert rg["nvoid"] == ro["vf"]["nvoid"]
    for k in rg["cubes"]:
        assert np.array_equal(rg["cubes"][k], ro["vf"]["cubes"][k]), k
    for k in ("indice", "uvoid", "ncellv", "marca", "volnew", "req", "gxc", "gyc", "gzc", "eps", "ip", "umean",
              "mtot"):
        assert np.array_equal(np.asarray(rg["cat"][k]), np.asarray(ro["cat"][k])), k


def test_grid_level_above_zero_rejected(gpu):
    from avism_b200.avism import AvismError
    u1, vs = grid_case(16)
    with pytest.raises(AvismError) as e:
        gpu.grid_fields(Params(nx=32, periodic=1, lado0=100.0, level=1), 16, u1, *vs)
    assert e.value.code == 8 and "BIN_GRID" in str(e.value)
