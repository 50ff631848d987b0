"""MASCLET input (FLAG_DATA = 0) on the CPU: the library's reader of the grid,
gas and dark-matter files (READ_MASCLET, src/reader.f90:86-405) against the
values written, and the oracle's level fields (src/avism.f90:980-1156,
1366-1405, 1633-1650) against a numpy restatement of the FLAG_DENS / FLAG_DIV
combinations built from the oracle's own interpolation and DIVER_UNIFORM; at
level 1 the oracle's DIVER_FINA_GAS + VMESH against a numpy restatement, and
its refusals of patches that reach outside the reference's arrays."""
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


def test_reader_reads_the_level1_patches(tmp_path, snap):
    from avism_b200.avism import read_masclet_files
    r = read_masclet_files(*mc.write_files(snap, str(tmp_path)), snap["ng"])
    want = mc.amr(snap)
    assert set(r["amr"]) == set(want)
    for k in want:
        assert np.array_equal(r["amr"][k], want[k]), k


def _amr_level1_np(p, nh, u1g, u2g, u3g, u4g, a):
    """UGR and DIVR of DIVER_FINA_GAS (src/divergence.f90:140-340) and VMESH
    (src/amr2uniform.f90:127-248) restated with numpy REAL*4 arrays [k, j, i]."""
    f32 = np.float32
    g, rad = O.grid_setup(p)
    g0, _ = O.grid_setup(Params(nx=nh, periodic=p.periodic, lado0=p.lado0, level=0))
    dx0, dxr, rx1, nx = f32(g0.dx), f32(g.dx), f32(rad[1 - g.rad_lo]), g.nx
    h0, hr = f32(f32(2.0) * dx0), f32(f32(2.0) * f32(dx0 / f32(2.0)))
    U = [np.asarray(v, f32).reshape(nh, nh, nh) for v in (u1g, u2g, u3g, u4g)]
    dint = np.zeros((nh, nh, nh), f32)
    c = slice(1, -1)
    dint[c, c, c] = ((U[1][c, c, 2:] - U[1][c, c, :-2]) / h0 + (U[2][c, 2:, c] - U[2][c, :-2, c]) / h0) + \
        (U[3][2:, c, c] - U[3][:-2, c, c]) / h0
    d0 = dint.copy()
    d0[:, :, 0] = d0[:, :, 1]
    d0[:, :, -1] = d0[:, :, -2]
    d0[:, 0, :] = d0[:, 1, :]
    d0[:, -1, :] = d0[:, -2, :]
    d0[0] = d0[1]
    d0[-1] = d0[-2]
    flag = np.ones((nx, nx, nx), np.int32)
    ugr = np.zeros((nx, nx, nx), f32)
    divr = np.zeros((nx, nx, nx), f32)
    flagr = np.zeros((nh, nh, nh), bool)
    for q in range(len(a["nx"])):
        n1, n2, n3 = (int(a[k][q]) for k in ("nx", "ny", "nz"))
        l1, l2, l3 = (int(a[k][q]) for k in ("ix", "iy", "iz"))
        sl = slice(int(a["offset"][q]), int(a["offset"][q + 1]))
        V = [np.asarray(a[k][sl], f32).reshape(n3, n2, n1) for k in ("u11g", "u12g", "u13g", "u14g")]
        own = np.zeros((n3, n2, n1), f32)
        own[c, c, c] = ((V[1][c, c, 2:] - V[1][c, c, :-2]) / hr + (V[2][c, 2:, c] - V[2][c, :-2, c]) / hr) + \
            (V[3][2:, c, c] - V[3][:-2, c, c]) / hr
        kk, jj, ii = np.meshgrid(np.arange(1, n3 + 1), np.arange(1, n2 + 1), np.arange(1, n1 + 1), indexing="ij")
        rim = (ii < 3) | (ii > n1 - 2) | (jj < 3) | (jj > n2 - 2) | (kk < 3) | (kk > n3 - 2)
        aux = np.where(rim, dint[(kk + 1) // 2 + l3 - 2, (jj + 1) // 2 + l2 - 2, (ii + 1) // 2 + l1 - 2], f32(0))
        two = (ii == 2) | (ii == n1 - 1) | (jj == 2) | (jj == n2 - 1) | (kk == 2) | (kk == n3 - 1)
        one = (ii == 1) | (ii == n1) | (jj == 1) | (jj == n2) | (kk == 1) | (kk == n3)
        dv = np.where(two, (f32(0.5) * (aux + own)).astype(f32), own)
        dv = np.where(one, aux, dv)
        r1 = [int(f32(f32(f32(a[k][q]) - f32(f32(0.5) * dxr)) - rx1) / dxr + f32(0.5)) for k in ("rx", "ry", "rz")]
        box = (slice(r1[2], r1[2] + n3), slice(r1[1], r1[1] + n2), slice(r1[0], r1[0] + n1))
        flag[box] += 1
        ugr[box] = ugr[box] + V[0]
        divr[box] = divr[box] + dv
        flagr[r1[2] // 2:(r1[2] + n3 - 1) // 2 + 1, r1[1] // 2:(r1[1] + n2 - 1) // 2 + 1,
              r1[0] // 2:(r1[0] + n1 - 1) // 2 + 1] = True
    ugr = (ugr / flag.astype(f32)).astype(f32)
    divr = (divr / flag.astype(f32)).astype(f32)
    up = lambda b: b.repeat(2, 0).repeat(2, 1).repeat(2, 2)
    keep = up(flagr)
    return np.where(keep, ugr, up(U[0])).ravel(), np.where(keep, divr, up(d0)).ravel()


@pytest.mark.parametrize("fd,fv", [(2, 2), (0, 0), (1, 1), (2, -1), (0, 2)])
def test_oracle_level1(snap, fd, fv):
    ng = snap["ng"]
    p = Params(nx=2 * ng, periodic=1, lado0=snap["box"], level=1, levmin=1, flag_dens=fd, flag_div=fv)
    parts = mc.particles(snap)
    u1e, dve, md = O.masclet_fields(p, ng, mc.gas(snap), parts, mc.amr(snap))
    ugr, divr = _amr_level1_np(p, ng, *mc.gas(snap), mc.amr(snap))
    f32 = np.float32
    g, _ = O.grid_setup(p)
    if fd <= 1:
        r = O.particles_to_grid(p, *(parts[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
        vol = f32(f32(f32(g.dx * g.dx) * g.dx) * f32(f32(g.rete * g.rete) * g.rete))
        dm = ((r["u_mass"] / vol).astype(f32) / f32(g.rote)).astype(f32)
    u = {0: (dm + ugr).astype(f32) if fd == 0 else None, 1: dm if fd == 1 else None, 2: ugr}[fd]
    u1 = (u * f32(g.rote)).astype(f32)
    mean = f32(np.cumsum(u1.astype(np.float64))[-1] / u1.size)
    u1 = (u1 / mean).astype(f32)
    assert np.array_equal(_inner(p, u1e), u1)
    if fv == -1:
        coef = f32(f32(f32(np.power(f32(p.omega0), f32(0.6))) * f32(g.rete)) * f32(g.hte))
        dv = (-(coef * (u1 - f32(1.0)))).astype(f32)
    else:                                           # DIVERDMCO = 0 above level 0
        dv = {0: np.where(f32(0) < divr, f32(0), divr), 1: np.zeros_like(divr), 2: divr}[fv]
    assert np.array_equal(_inner(p, dve), dv)
    assert md > 0


def test_oracle_level1_without_patches_is_the_base_grid(snap):
    ng = snap["ng"]
    p = Params(nx=2 * ng, periodic=1, lado0=snap["box"], level=1, levmin=1, flag_dens=2, flag_div=2)
    none = {k: np.zeros(0, np.int32) for k in ("nx", "ny", "nz", "ix", "iy", "iz")}
    none.update({k: np.zeros(0, np.float32) for k in ("rx", "ry", "rz", "u11g", "u12g", "u13g", "u14g")})
    none["offset"] = np.zeros(1, np.int64)
    u1e, dve, _ = O.masclet_fields(p, ng, mc.gas(snap), None, none)
    ugr, divr = _amr_level1_np(p, ng, *mc.gas(snap), none)
    up = mc.gas(snap)[0].reshape(ng, ng, ng).repeat(2, 0).repeat(2, 1).repeat(2, 2).ravel()
    assert np.array_equal(ugr, up)
    assert np.array_equal(_inner(p, dve), divr)


@pytest.mark.parametrize("bad", ["rim", "vmesh", "offset", "nan", "huge", "edge"])
def test_oracle_level1_rejects_patches_outside(snap, bad):
    ng = snap["ng"]
    p = Params(nx=2 * ng, periodic=1, lado0=snap["box"], level=1, levmin=1, flag_dens=2, flag_div=2)
    a = {k: np.array(v, copy=True) for k, v in mc.amr(snap).items()}
    if bad == "rim":
        a["ix"][0] = 1                              # the rim's parent differences need U2G(0)
    elif bad == "vmesh":
        a["rz"][2] = a["rz"][2] + np.float32(40 * 2.0)    # the patch lands beyond the level grid
    elif bad == "offset":
        a["offset"][1] += 1
    elif bad == "nan":
        a["rx"][1] = np.float32(np.nan)                 # INT() of it is undefined
    elif bad == "huge":
        a["ry"][0] = np.float32(1e30)
    else:
        a["nx"][0] = np.int32(2 ** 21)                  # a size product beyond any grid
    with pytest.raises(O.OracleError):
        O.masclet_fields(p, ng, mc.gas(snap), None, a)


def test_oracle_level_above_one_is_unsupported(snap):
    p = Params(nx=4 * snap["ng"], periodic=1, lado0=snap["box"], level=2)
    with pytest.raises(O.OracleError):
        O.masclet_fields(p, snap["ng"], mc.gas(snap), mc.particles(snap))


def test_oracle_gas_only_needs_no_particles(snap):
    p = Params(nx=snap["ng"] // 2, periodic=0, lado0=snap["box"], level=-1, levmin=-1, flag_dens=2, flag_div=2)
    u1, dv, md = O.masclet_fields(p, snap["ng"], mc.gas(snap), None)
    assert np.isfinite(u1).all() and np.isfinite(dv).all() and md > 0


def test_oracle_level1_inside_level0_voids(snap):
    """Voids-in-voids on MASCLET input: level 0, its parent map (next_level),
    then level 1 from the patches inside the level-0 voids; every level-1 cube
    has a level-0 father."""
    ng = snap["ng"]
    p0 = Params(nx=ng, periodic=1, lado0=snap["box"], level=0, levmin=0, flag_dens=2, flag_div=2)
    o0 = O.run_level_masclet(p0, ng, mc.gas(snap), None)
    mp, rq = O.next_level(p0, o0["vf"]["nvoid"], o0["cat"]["marca"], o0["cat"]["uvoid"], o0["cat"]["req"])
    assert 0 < np.mean(mp > 0) < 1
    p1 = Params(nx=2 * ng, periodic=1, lado0=snap["box"], level=1, levmin=0, flag_dens=2, flag_div=2)
    o1 = O.run_sublevel_masclet(p1, ng, mc.gas(snap), mp, rq, None, mc.amr(snap))
    assert o1["vf"]["nvoid"] > 0 and o1["cat"]["nvoidt"] > 0
    assert np.all(np.asarray(o1["vf"]["cubes"]["father"]) > 0)


def test_patch_reader_rejects_short_files_and_small_capacities(tmp_path, snap):
    """The level-1 patch reader: a gas file cut inside the first patch's
    records is an I/O error; capacities below the patch or cell counts are
    refused before anything is written."""
    import ctypes as C
    from avism_b200 import _lib
    from avism_b200.avism import AvismError, read_masclet_patches
    grid, gas, dm = mc.write_files(snap, str(tmp_path))
    ng3 = snap["ng"] ** 3
    base = (8 + 8) + 10 * (8 + 4 * ng3)            # header + the ten level-0 records
    with open(gas, "rb") as f:
        b = f.read()
    short = str(tmp_path / "gas_short")
    with open(short, "wb") as f:
        f.write(b[:base + 100])
    with pytest.raises(AvismError):
        read_masclet_patches(grid, short, snap["ng"])
    lib = _lib.load()
    npatch, ncells = C.c_int32(), C.c_int64()
    assert lib.avism_io_masclet_patches_size(grid.encode(), C.byref(npatch), C.byref(ncells)) == 0
    want = mc.amr(snap)
    assert npatch.value == len(want["nx"]) and ncells.value == len(want["u11g"])
    arrs = [np.zeros(16, np.int32) for _ in range(6)] + [np.zeros(16, np.float32) for _ in range(3)] + \
        [np.zeros(17, np.int64)] + [np.zeros(ncells.value, np.float32) for _ in range(4)]
    ptrs = [a.ctypes.data_as(C.c_void_p) for a in arrs]
    args = (grid.encode(), gas.encode(), snap["ng"])
    assert lib.avism_io_read_masclet_patches(*args, npatch.value - 1, ncells.value, *ptrs) != 0
    assert lib.avism_io_read_masclet_patches(*args, npatch.value, ncells.value - 1, *ptrs) != 0
    assert lib.avism_io_read_masclet_patches(*args, npatch.value, ncells.value, *ptrs) == 0
    assert np.array_equal(arrs[-4], want["u11g"])

