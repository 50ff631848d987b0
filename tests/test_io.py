"""The on-disk formats at the boundary (host only, no GPU): the particle file
of READ_BINARY_PART_1 and the voids / cubes / map files of one iteration,
checked by reading them back as tools/read_voids.py does (and with that tool
itself when the reference is mounted)."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from avism_b200 import _lib, synth
from avism_b200._abi import Params
from avism_b200.avism import (AvismError, append_catalogue_level, read_particle_file,
                              write_catalogue_headers)
from oracle import oracle as O

# tools/read_voids.py of the reference checkout named by AVISM_REFERENCE_ROOT
# (unset: the test that runs the tool is skipped)
_REF = os.environ.get("AVISM_REFERENCE_ROOT")
READ_VOIDS = os.path.join(_REF, "tools", "read_voids.py") if _REF else ""


def _fortran_records(path, records):
    """Fortran sequential unformatted: each record framed by its byte length."""
    with open(path, "wb") as f:
        for r in records:
            b = r.tobytes() if hasattr(r, "tobytes") else r
            f.write(np.uint32(len(b)).tobytes() + b + np.uint32(len(b)).tobytes())


def test_particle_file_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    n = 1000
    cols = [rng.uniform(-50, 50, n).astype(np.float32) for _ in range(3)] + \
           [rng.normal(0, 300, n).astype(np.float32) for _ in range(3)] + [np.full(n, 1e10, np.float32)]
    path = tmp_path / "bin_file_part00001"
    _fortran_records(path, [np.int64(n).tobytes() + np.float32(0.5).tobytes()] + cols)
    r = read_particle_file(path)
    assert r["zeta"] == np.float32(0.5)
    for k, c in zip(("x", "y", "z", "vx", "vy", "vz", "m"), cols):
        assert np.array_equal(r[k], c), k


def test_particle_file_errors(tmp_path):
    lib = _lib.load()
    n = 10
    path = tmp_path / "p"
    cols = [np.zeros(n, np.float32)] * 7
    _fortran_records(path, [np.int64(n).tobytes() + np.float32(0.0).tobytes()] + cols)
    bufs = [np.zeros(n, np.float32) for _ in range(7)]
    ptrs = [C.c_void_p(b.ctypes.data) for b in bufs]
    assert lib.avism_io_read_particles(os.fsencode(path), n - 1, *ptrs) == 1       # NPARTT > capacity
    bad = tmp_path / "bad"
    _fortran_records(bad, [np.int64(n).tobytes() + np.float32(0.0).tobytes()] + cols[:6] + [np.zeros(n - 1,
                                                                                                 np.float32)])
    assert lib.avism_io_read_particles(os.fsencode(bad), n, *ptrs) == 10            # short last record
    with pytest.raises(AvismError):
        read_particle_file(tmp_path / "missing")


@pytest.fixture(scope="module")
def level():
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=64.0, nsph=3, rmin=5.0, rmax=9.0, seed=7))
    p = Params(nx=32, periodic=1, lado0=64.0)
    r = O.run_level(p, parts)
    res = dict(cubes=r["vf"]["cubes"], nvoid=r["vf"]["nvoid"], cat=r["cat"], meandens=r["meandens"])
    return p, res, r["u1co"], r["diverco"]


def _read_voids_file(path):
    """The parse of read_void_catalogue (tools/read_voids.py)."""
    with open(path) as f:
        h = f.readline().split()
        head = dict(nlev=int(h[0]), levmin=int(h[1]), levmax=int(h[2]), nmax=int(h[3]), L0=float(h[6]))
        levels = []
        for _ in range(head["nlev"]):
            lev, ncubes, nvoids, nparents, ff, md = f.readline().split()
            rows = [np.array(f.readline().split()).astype("f4") for _ in range(int(nvoids))]
            levels.append(dict(level=int(lev), ncubes=int(ncubes), nvoids=int(nvoids), nparents=int(nparents),
                               FF=float(ff), meandens=float(md), rows=np.array(rows)))
    return head, levels


def test_catalogue_cubes_and_map_files(tmp_path, level):
    p, res, u1, dv = level
    cat, cubes, nv = res["cat"], res["cubes"], res["nvoid"]
    vp, cp, mp = tmp_path / "voids00001", tmp_path / "cubes00001", tmp_path / "map00001"
    write_catalogue_headers(vp, cp, 1, 0, 0, 32, 32, 32, 64.0)
    append_catalogue_level(vp, p, res, cubes_path=cp, map_path=mp, u1co_ext=u1, diverco_ext=dv)
    head, levels = _read_voids_file(vp)
    assert head == dict(nlev=1, levmin=0, levmax=0, nmax=32, L0=64.0)
    lv = levels[0]
    main = [i - 1 for i in cat["indice"] if cat["uvoid"][i - 1] == -1]
    assert (lv["level"], lv["ncubes"], lv["nvoids"], lv["nparents"]) == (0, nv, cat["nvoidt"], 0) and main
    assert lv["meandens"] == pytest.approx(res["meandens"], rel=1e-7)
    assert lv["FF"] == pytest.approx(cat["volt_clean"] / np.float32(64.0) ** 3, rel=1e-15)
    rows = lv["rows"]
    assert np.array_equal(rows[:, 0], np.array(main) + 1)
    for col, k in enumerate(("xc", "yc", "zc", "gxc", "gyc", "gzc", "volnew", "req", "umean", "eps", "ip"), 1):
        assert np.array_equal(rows[:, col], cat[k][main]), k
    assert np.all(rows[:, 12] == 0) and np.all(rows[:, 13] == 0)       # no parent at LEVMIN
    assert np.array_equal(rows[:, 14], cat["mtot"][main])
    # cubes: every cube in INDICE order
    lines = open(cp).read().split("\n")
    assert lines[0].split() == ["1", "0", "0"] and lines[1].split() == ["0", str(nv), str(cat["nvoidt"])]
    for iv, line in enumerate(lines[2:2 + nv]):
        i = cat["indice"][iv] - 1
        t = line.split()
        assert int(t[0]) == i + 1 and int(t[1]) == cat["uvoid"][i]
        assert [int(v) for v in t[2:8]] == [int(cubes[k][i]) for k in ("inicio_x", "final_x", "inicio_y",
                                                                       "final_y", "inicio_z", "final_z")]
        assert np.array_equal(np.array(t[8:], "f4"), np.array([cubes[k][i] for k in (
            "rini_x", "rfin_x", "rini_y", "rfin_y", "rini_z", "rfin_z")], np.float32))
    # map: inner MARCA, U1CO - 1, DIVERCO, column-major
    g, _ = O.grid_setup(p)
    o, nx, ne = 1 - g.low1, g.nx, g.ne
    inner = lambda a: np.asarray(a).reshape((ne, ne, ne), order="F")[o:o + nx, o:o + nx, o:o + nx]
    with open(mp, "rb") as f:
        marca = np.fromfile(f, np.int32, nx ** 3).reshape((nx,) * 3, order="F")
        delta = np.fromfile(f, np.float32, nx ** 3).reshape((nx,) * 3, order="F")
        div = np.fromfile(f, np.float32, nx ** 3).reshape((nx,) * 3, order="F")
        assert f.read() == b""
    assert np.array_equal(marca, inner(cat["marca"]))
    assert np.array_equal(delta, np.float32(-1.0) + inner(u1))
    assert np.array_equal(div, inner(dv))


def test_sublevel_parent_columns(tmp_path, level):
    """Above LEVMIN: INDP = FATHER(IND) and REQPP = the parent's REQ."""
    p, res, _, _ = level
    nv = res["nvoid"]
    rng = np.random.default_rng(2)
    cubes = {k: np.array(v) for k, v in res["cubes"].items()}
    cubes["father"] = rng.integers(1, 6, nv).astype(np.int32)
    req_parent = np.array([1.5, 2.5, 3.5, 4.5, 5.5], np.float32)
    sub = dict(res, cubes=cubes)
    q = Params(nx=32, periodic=1, lado0=64.0, level=1, levmin=0)
    vp = tmp_path / "voids00001"
    write_catalogue_headers(vp, None, 1, 0, 1, 32, 32, 32, 64.0)
    append_catalogue_level(vp, q, sub, nvoidp=5, req_parent=req_parent)
    _, levels = _read_voids_file(vp)
    rows, cat = levels[0]["rows"], res["cat"]
    main = [i - 1 for i in cat["indice"] if cat["uvoid"][i - 1] == -1]
    assert levels[0]["level"] == 1 and levels[0]["nparents"] == 5
    assert np.array_equal(rows[:, 12], cubes["father"][main])
    assert np.array_equal(rows[:, 13], req_parent[cubes["father"][main] - 1])


@pytest.mark.skipif(not (READ_VOIDS and os.path.exists(READ_VOIDS)),
                    reason="AVISM_REFERENCE_ROOT does not name a reference checkout with tools/read_voids.py")
def test_reference_reader_reads_the_files(tmp_path, level):
    """tools/read_voids.py itself parses the voids, cubes and map files."""
    p, res, u1, dv = level
    vp, cp, mp = tmp_path / "voids00001", tmp_path / "cubes00001", tmp_path / "map00001"
    write_catalogue_headers(vp, cp, 1, 0, 0, 32, 32, 32, 64.0)
    append_catalogue_level(vp, p, res, cubes_path=cp, map_path=mp, u1co_ext=u1, diverco_ext=dv)
    spec = importlib.util.spec_from_file_location("read_voids", READ_VOIDS)
    rv = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rv)
    details, levels = rv.read_void_catalogue(1, str(tmp_path), output_format="arrays")
    cat = res["cat"]
    main = [i - 1 for i in cat["indice"] if cat["uvoid"][i - 1] == -1]
    assert details["nmax"] == 32 and levels[0]["nvoids"] == cat["nvoidt"]
    assert np.array_equal(levels[0]["voids"]["R"], cat["req"][main])
    assert np.array_equal(levels[0]["voids"]["M"], cat["mtot"][main])
    cl = rv.read_cubes(1, str(tmp_path), output_format="arrays")
    assert cl[0]["ncubes"] == res["nvoid"]
    marca, delta = rv.read_void_map(1, str(tmp_path), output_marca=True, output_deltaTot=True)
    g, _ = O.grid_setup(p)
    o, nx, ne = 1 - g.low1, g.nx, g.ne
    ext = np.asarray(cat["marca"]).reshape((ne,) * 3, order="F")
    assert np.array_equal(marca[0], ext[o:o + nx, o:o + nx, o:o + nx])


def _fortran_subrecords(f, payload, chunk):
    """One logical record written as gfortran's chain of subrecords of at most
    `chunk` bytes: a negative leading marker when another subrecord follows, a
    negative trailing marker on every subrecord after the first."""
    parts = [payload[i:i + chunk] for i in range(0, len(payload), chunk)] or [b""]
    for i, part in enumerate(parts):
        head = -len(part) if i < len(parts) - 1 else len(part)
        tail = -len(part) if i > 0 else len(part)
        f.write(np.int32(head).tobytes() + part + np.int32(tail).tobytes())


def test_particle_file_with_split_records(tmp_path):
    """Records written as subrecord chains (gfortran splits records above
    2147483639 bytes) read back as the whole record."""
    rng = np.random.default_rng(3)
    n = 777
    cols = [rng.normal(0, 10, n).astype(np.float32) for _ in range(7)]
    path = tmp_path / "split"
    with open(path, "wb") as f:
        _fortran_subrecords(f, np.int64(n).tobytes() + np.float32(1.5).tobytes(), 12)
        for i, c in enumerate(cols):
            _fortran_subrecords(f, c.tobytes(), [4, 1000, 3108, 400, 1, 7, 64][i])
    r = read_particle_file(path)
    assert r["zeta"] == np.float32(1.5)
    for k, c in zip(("x", "y", "z", "vx", "vy", "vz", "m"), cols):
        assert np.array_equal(r[k], c), k
    bad = tmp_path / "badsplit"                      # chain whose trailing marker lies
    with open(bad, "wb") as f:
        _fortran_subrecords(f, np.int64(n).tobytes() + np.float32(1.5).tobytes(), 12)
        b = cols[0].tobytes()
        f.write(np.int32(-100).tobytes() + b[:100] + np.int32(-99).tobytes())
    lib = _lib.load()
    bufs = [np.zeros(n, np.float32) for _ in range(7)]
    assert lib.avism_io_read_particles(os.fsencode(bad), n, *(C.c_void_p(b.ctypes.data) for b in bufs)) == 10


def test_particle_file_without_velocities(tmp_path):
    from avism_b200.avism import read_particle_file_novel
    rng = np.random.default_rng(4)
    n = 500
    cols = [rng.uniform(-50, 50, n).astype(np.float32) for _ in range(3)] + [np.full(n, 3e9, np.float32)]
    path = tmp_path / "bin_file_part2"
    _fortran_records(path, [np.int64(n).tobytes() + np.float32(0.25).tobytes()] + cols)
    r = read_particle_file_novel(path)
    assert r["zeta"] == np.float32(0.25) and set(r) == {"x", "y", "z", "m", "zeta"}
    for k, c in zip(("x", "y", "z", "m"), cols):
        assert np.array_equal(r[k], c), k


def test_grid_file(tmp_path):
    from avism_b200.avism import read_grid_file
    rng = np.random.default_rng(5)
    nx = 12
    grids = [rng.normal(0, 1, nx ** 3).astype(np.float32) for _ in range(4)]
    path = tmp_path / "bin_file_grid00001"
    _fortran_records(path, [np.float32(0.0).tobytes()] + grids)
    r = read_grid_file(path, nx)
    for k, g in zip(("u1", "u2", "u3", "u4"), grids):
        assert np.array_equal(r[k], g), k
    with pytest.raises(AvismError):
        read_grid_file(path, nx + 1)                  # records shorter than (nx+1)^3


def test_mask_file_maps_to_level(tmp_path):
    """mask.dat at the coarse grid, mapped onto a level 4x finer by integer
    refinement; positive values become 1, zero and negative ones stay."""
    from avism_b200.avism import read_mask_file
    rng = np.random.default_rng(6)
    nm = 8
    m2 = rng.integers(-2, 4, nm ** 3).astype(np.int8)
    path = tmp_path / "mask.dat"
    with open(path, "wb") as f:
        f.write(np.int32(nm).tobytes() + np.array([-1.0, 1.0, 2.0], np.float32).tobytes() + m2.tobytes())
    sm, lims = read_mask_file(path, nm, nm)
    assert np.array_equal(lims, np.array([-1.0, 1.0, 2.0], np.float32))
    assert np.array_equal(sm, np.where(m2 > 0, 1, m2).astype(np.int8))
    fine, _ = read_mask_file(path, nm, 4 * nm)
    m3 = np.where(m2 > 0, 1, m2).reshape(nm, nm, nm)                     # [k][j][i]
    want = m3.repeat(4, 0).repeat(4, 1).repeat(4, 2).ravel()
    assert np.array_equal(fine, want)
    with pytest.raises(AvismError):
        read_mask_file(path, nm + 1, nm + 1)          # 'MASK grid does not coincide'
    with pytest.raises(AvismError):
        read_mask_file(path, nm, 3 * nm)              # odd refinement


def test_randoms_file_and_vel_cube(tmp_path):
    from avism_b200.avism import read_randoms_file, write_vel_cube
    rng = np.random.default_rng(7)
    n = 321
    cols = [rng.uniform(-9, 9, n).astype(np.float32) for _ in range(3)] + [rng.uniform(0.5, 2, n).astype(np.float32)]
    path = tmp_path / "rands.dat"
    _fortran_records(path, [np.int32(n).tobytes()] + cols)
    r = read_randoms_file(path)
    for k, c in zip(("x", "y", "z", "w"), cols):
        assert np.array_equal(r[k], c), k
    nx = 6
    g = [rng.normal(0, 1, nx ** 3).astype(np.float32) for _ in range(3)]
    vp = tmp_path / "vel_cube.dat"
    write_vel_cube(vp, nx, *g)
    raw = np.fromfile(vp, np.float32)
    assert np.array_equal(raw, np.concatenate(g))
