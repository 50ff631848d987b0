"""Grid input (FLAG_DATA = 2, READ_BINARY_GRID) on the CPU: the oracle's
SMOOTH_2 (src/amr2uniform.f90:65-120) is the block average of the input grid
for levels below 0, the mean of rho/rho_B is kept, and a grid file read with the
library's reader runs through a whole level."""
import numpy as np
import pytest

from avism_b200 import synth
from avism_b200._abi import Params, UV
from oracle import oracle as O


def grid_case(ng=64, seed=3):
    """delta + 1 of a lognormal field and linear-theory velocities (/ UV), column-major."""
    rng = np.random.default_rng(seed)
    g, vel = synth._grf(ng, 100.0, -1.5, 1.0, rng)
    rho = np.exp(g)
    rho /= rho.mean()
    cm = lambda a: np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()
    u1 = cm(rho).astype(np.float32)
    vs = [(cm(v * 300.0 / np.std(v)).astype(np.float32) / np.float32(UV)).astype(np.float32) for v in vel]
    return u1, vs


@pytest.mark.parametrize("lev", [-1, -2])
def test_smooth2_is_the_block_average(lev):
    u1, vs = grid_case()
    f = 2 ** -lev
    nx = 64 // f
    p = Params(nx=nx, periodic=0, lado0=100.0, level=lev, levmin=lev)
    got, _, _ = O.grid_fields(p, 64, u1, *vs)
    want = u1.astype(np.float64).reshape(nx, f, nx, f, nx, f).mean(axis=(1, 3, 5)).ravel()
    assert np.allclose(got, want, rtol=2e-6, atol=0)


def test_level_above_zero_is_the_reference_stop():
    u1, vs = grid_case(16)
    with pytest.raises(O.OracleError) as e:
        O.grid_fields(Params(nx=32, periodic=1, lado0=100.0, level=1), 16, u1, *vs)
    assert "8" in str(e.value)


def test_grid_file_level(tmp_path):
    from avism_b200.avism import read_grid_file
    u1, vs = grid_case(32)
    path = tmp_path / "bin_file_grid00001"
    delta = (u1 - np.float32(1)).astype(np.float32)
    kms = [(v * np.float32(UV)).astype(np.float32) for v in vs]
    with open(path, "wb") as f:
        for rec in [np.float32(0.0).tobytes()] + [a.tobytes() for a in [delta] + kms]:
            f.write(np.uint32(len(rec)).tobytes() + rec + np.uint32(len(rec)).tobytes())
    r = read_grid_file(path, 32)
    # the reference's conversions after reading (src/reader.f90:546-550)
    g1 = (r["u1"] + np.float32(1.0)).astype(np.float32)
    gv = [(r[k] / np.float32(UV)).astype(np.float32) for k in ("u2", "u3", "u4")]
    p = Params(nx=32, periodic=1, lado0=100.0, rmin=2.0)
    a = O.run_level_grid(p, 32, g1, *gv)
    b = O.run_level_grid(p, 32, u1, *vs)
    assert a["vf"]["nvoid"] == b["vf"]["nvoid"] > 0
    assert np.array_equal(a["cat"]["marca"], b["cat"]["marca"])
