"""MASCLET input (FLAG_DATA = 0) on the CPU: the library's reader of the grid,
gas and dark-matter files (READ_MASCLET, src/reader.f90:86-405) against the
values written, and the oracle's level fields (src/avism.f90:980-1156,
1366-1405, 1633-1650) against a numpy restatement of the FLAG_DENS / FLAG_DIV
combinations built from the oracle's own interpolation and DIVER_UNIFORM."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O

import masclet_case as mc


@pytest.fixture(scope="module")
def snap():
    return mc.snapshot()


def test_reader_reads_what_was_written(tmp_path, snap):
    from avism_b200.avism import read_masclet_files
    paths = mc.write_files(snap, str(tmp_path), zeta=0.25)
    r = read_masclet_files(*paths, snap["ng"])
    assert r["nl"] == 2 and r["ndxyz0"] == len(snap["lev0"]["x"])
    assert r["zeta"] == np.float32(0.25) and r["map"] == snap["map"]
    for got, want in zip((r["gas"][k] for k in ("u1g", "u2g", "u3g", "u4g")), mc.gas(snap)):
        assert np.array_equal(got, want)
    want = mc.particles(snap)
    for k in want:
        assert np.array_equal(r["parts"][k], want[k]), k


def test_reader_rejects_a_short_file(tmp_path, snap):
    import os
    from avism_b200.avism import AvismError, read_masclet_files
    grid, gas, dm = mc.write_files(snap, str(tmp_path))
    with open(dm, "rb") as f:
        b = f.read()
    with open(dm, "wb") as f:
        f.write(b[: len(b) - 100])
    with pytest.raises(AvismError):
        read_masclet_files(grid, gas, dm, snap["ng"])
    assert os.path.getsize(dm) == len(b) - 100


def _inner(p, ext):
    g, _ = O.grid_setup(p)
    o = 1 - g.low1
    n = g.nx
    return ext.reshape(g.ne, g.ne, g.ne)[o:o + n, o:o + n, o:o + n].ravel()


@pytest.mark.parametrize("fd,fv", [(0, 0), (1, 1), (2, 2), (0, -1), (2, 1), (1, 2)])
def test_oracle_combinations(snap, fd, fv):
    p = Params(nx=snap["ng"], periodic=1, lado0=snap["box"], flag_dens=fd, flag_div=fv)
    parts = mc.particles(snap)
    u1g, u2g, u3g, u4g = mc.gas(snap)
    u1e, dve, md = O.masclet_fields(p, snap["ng"], (u1g, u2g, u3g, u4g), parts)
    # the restatement: DM grids from the oracle's interpolation, then the REAL*4 steps
    r = O.particles_to_grid(p, *(parts[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
    g, _ = O.grid_setup(p)
    f32 = np.float32
    vol = f32(f32(f32(g.dx * g.dx) * g.dx) * f32(f32(g.rete * g.rete) * g.rete))
    dm = (r["u_mass"] / vol).astype(f32)
    dm = (dm / f32(g.rote)).astype(f32)
    u = {0: (dm + u1g).astype(f32), 1: dm, 2: u1g}[fd]
    u1 = (u * f32(g.rote)).astype(f32)
    mean = f32(np.cumsum(u1.astype(np.float64))[-1] / u1.size)       # sequential REAL*8 sum
    u1 = (u1 / mean).astype(f32)
    assert np.array_equal(_inner(p, u1e), u1)
    if fv == -1:
        coef = f32(f32(f32(np.power(f32(p.omega0), f32(0.6))) * f32(g.rete)) * f32(g.hte))
        dv = (-(coef * (u1 - f32(1.0)))).astype(f32)
    else:
        dg = O.diver_uniform(p.nx, g.dx, u2g, u3g, u4g, p.periodic)
        dd = O.diver_uniform(p.nx, g.dx, r["u2"], r["u3"], r["u4"], p.periodic)
        dv = {0: np.where(dd < dg, dd, dg), 1: dd, 2: dg}[fv]
    assert np.array_equal(_inner(p, dve), dv)
    assert md > 0


def test_oracle_level_above_zero_is_unsupported(snap):
    p = Params(nx=2 * snap["ng"], periodic=1, lado0=snap["box"], level=1)
    with pytest.raises(O.OracleError):
        O.masclet_fields(p, snap["ng"], mc.gas(snap), mc.particles(snap))


def test_oracle_gas_only_needs_no_particles(snap):
    p = Params(nx=snap["ng"] // 2, periodic=0, lado0=snap["box"], level=-1, levmin=-1, flag_dens=2, flag_div=2)
    u1, dv, md = O.masclet_fields(p, snap["ng"], mc.gas(snap), None)
    assert np.isfinite(u1).all() and np.isfinite(dv).all() and md > 0
