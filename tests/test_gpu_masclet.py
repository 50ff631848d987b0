"""GPU parity for MASCLET input (FLAG_DATA = 0) at levels 1, 0 and -1: the
level's U1CO / DIVERCO and whole catalogue through the C-ABI against the oracle,
bit for bit, for the FLAG_DENS / FLAG_DIV choices (src/avism.f90:1094-1124,
1366-1405, 1633-1650); level 1 from the AMR patches (DIVER_FINA_GAS, VMESH); a
snapshot read from its three files; patches outside the reference's arrays and
levels above 1 refused."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O

import masclet_case as mc

pytestmark = pytest.mark.gpu

CASES = [(0, 0, 0), (1, 1, 0), (2, 2, 0), (0, -1, 0), (0, 0, -1), (2, 2, -1), (2, 1, -1),
         (0, 0, 1), (2, 2, 1), (1, 1, 1), (2, -1, 1), (0, 2, 1)]


@pytest.fixture(scope="module")
def snap():
    return mc.snapshot()


def params(s, fd, fv, lev, periodic=1):
    nx = 2 * s["ng"] if lev == 1 else s["ng"] >> (-lev)
    return Params(nx=nx, periodic=periodic, lado0=s["box"], level=lev, levmin=lev, flag_dens=fd, flag_div=fv)


@pytest.mark.parametrize("fd,fv,lev", CASES)
def test_fields_and_level_exact(gpu, snap, fd, fv, lev):
    p = params(snap, fd, fv, lev)
    needs_dm = fd <= 1 or fv in (0, 1)
    parts = mc.particles(snap) if needs_dm else None
    amr = mc.amr(snap) if lev == 1 else None
    u1o, dvo, mdo = O.masclet_fields(p, snap["ng"], mc.gas(snap), parts, amr)
    u1g, dvg, mdg = gpu.masclet_fields(p, snap["ng"], mc.gas(snap), parts, amr)
    assert np.array_equal(u1o, u1g) and np.array_equal(dvo, dvg) and mdo == mdg
    o = O.run_level_masclet(p, snap["ng"], mc.gas(snap), parts, amr)
    g = gpu.run_level_masclet(p, snap["ng"], mc.gas(snap), parts, amr, capacity=200000)
    assert g["nvoid"] == o["vf"]["nvoid"]
    # at 16^3 the mock's voids fall below NCELL_MIN; at level 1 DIVERDMCO = 0
    # leaves MIN(DIVERGCO, 0) <= 0 (FLAG_DIV 0) or 0 (FLAG_DIV 1): no centres
    if lev == 0 or (lev == 1 and fv in (-1, 2)):
        assert g["nvoid"] > 0
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


def test_level1_from_files(gpu, snap, tmp_path):
    from avism_b200.avism import read_masclet_files
    r = read_masclet_files(*mc.write_files(snap, str(tmp_path)), snap["ng"])
    p = params(snap, 0, 0, 1)
    gas = tuple(r["gas"][k] for k in ("u1g", "u2g", "u3g", "u4g"))
    a = gpu.run_level_masclet(p, snap["ng"], gas, r["parts"], r["amr"], capacity=200000)
    o = O.run_level_masclet(p, snap["ng"], mc.gas(snap), mc.particles(snap), mc.amr(snap))
    assert a["nvoid"] == o["vf"]["nvoid"]
    for k in ("indice", "uvoid", "ncellv", "volnew", "umean", "mtot"):
        assert np.array_equal(a["cat"][k], o["cat"][k]), k


@pytest.mark.parametrize("bad", ["rim", "vmesh", "missing", "nan"])
def test_level1_refuses_patches_outside(gpu, snap, bad):
    """A patch whose rim needs base differences outside 2..NHY-1, or whose cells
    land outside the level grid, is refused (the kernels check every index
    before the access and report it); level 1 without patches too."""
    from avism_b200.avism import AvismError
    p = params(snap, 2, 2, 1)
    a = {k: np.array(v, copy=True) for k, v in mc.amr(snap).items()}
    if bad == "rim":
        a["ix"][0] = 1
    elif bad == "vmesh":
        a["rz"][2] = a["rz"][2] + np.float32(80.0)
    elif bad == "nan":
        a["rx"][1] = np.float32(np.nan)             # refused on the host, before any launch
    else:
        a = None
    with pytest.raises(AvismError):
        gpu.masclet_fields(p, snap["ng"], mc.gas(snap), None, a)
    # the context stays usable
    u1, dv, _ = gpu.masclet_fields(p, snap["ng"], mc.gas(snap), None, mc.amr(snap))
    u1o, dvo, _ = O.masclet_fields(p, snap["ng"], mc.gas(snap), None, mc.amr(snap))
    assert np.array_equal(u1, u1o) and np.array_equal(dv, dvo)


def test_level1_without_patches(gpu, snap):
    """No level-1 patches: every level-1 cell takes its base cell's U1G and
    DIVER0, as the oracle gives."""
    ng = snap["ng"]
    p = params(snap, 2, 2, 1)
    none = {k: np.zeros(0, np.int32) for k in ("nx", "ny", "nz", "ix", "iy", "iz")}
    none.update({k: np.zeros(0, np.float32) for k in ("rx", "ry", "rz", "u11g", "u12g", "u13g", "u14g")})
    none["offset"] = np.zeros(1, np.int64)
    u1o, dvo, mdo = O.masclet_fields(p, ng, mc.gas(snap), None, none)
    u1g, dvg, mdg = gpu.masclet_fields(p, ng, mc.gas(snap), None, none)
    assert np.array_equal(u1o, u1g) and np.array_equal(dvo, dvg) and mdo == mdg


@pytest.mark.parametrize("fd,fv", [(2, 2), (0, -1)])
def test_level1_inside_level0_voids(gpu, snap, fd, fv):
    """Voids-in-voids on MASCLET input, GPU against the oracle's same sequence:
    level 0, the parent map of next_level, level 1 from the patches inside the
    level-0 voids (cubes and catalogue bit-exact)."""
    ng = snap["ng"]
    parts = mc.particles(snap) if fd <= 1 else None
    p0 = params(snap, fd, fv, 0)
    o0 = O.run_level_masclet(p0, ng, mc.gas(snap), parts)
    g0 = gpu.run_level_masclet(p0, ng, mc.gas(snap), parts, want_marca=True, capacity=200000)
    assert np.array_equal(g0["cat"]["marca"], o0["cat"]["marca"])
    nv = o0["vf"]["nvoid"]
    mp, rq = O.next_level(p0, nv, o0["cat"]["marca"], o0["cat"]["uvoid"], o0["cat"]["req"])
    gmp, grq = gpu.next_level(p0, nv, g0["cat"]["marca"], g0["cat"]["uvoid"], g0["cat"]["req"])
    assert np.array_equal(mp, gmp) and np.array_equal(rq, grq)
    p1 = Params(nx=2 * ng, periodic=1, lado0=snap["box"], level=1, levmin=0, flag_dens=fd, flag_div=fv)
    o1 = O.run_sublevel_masclet(p1, ng, mc.gas(snap), mp, rq, parts, mc.amr(snap))
    g1 = gpu.run_sublevel_masclet(p1, ng, mc.gas(snap), mp, rq, parts, mc.amr(snap), want_marca=True,
                                  capacity=200000)
    assert g1["nvoid"] == o1["vf"]["nvoid"] > 0
    for k in g1["cubes"]:
        assert np.array_equal(g1["cubes"][k], o1["vf"]["cubes"][k]), k
    for k in ("indice", "uvoid", "ncellv", "marca", "volnew", "req", "gxc", "gyc", "gzc", "eps", "ip", "umean",
              "mtot"):
        assert np.array_equal(g1["cat"][k], o1["cat"][k]), k
    assert np.all(np.asarray(g1["cubes"]["father"]) > 0)


def test_level_above_one_is_unsupported(gpu, snap):
    from avism_b200.avism import AvismError
    p = Params(nx=4 * snap["ng"], periodic=1, lado0=snap["box"], level=2)
    with pytest.raises(AvismError) as e:
        gpu.masclet_fields(p, snap["ng"], mc.gas(snap), mc.particles(snap))
    assert "not implemented" in str(e.value)
