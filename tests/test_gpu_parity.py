"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle.

Bit-exact: kNN lists, INDEXX permutations, the SPH and TSC fields, normalised
density, divergence, flag grids, the grown cubes and every catalogue column
(the REAL*4 inertia, UMEAN and MTOT sums in the reference's serial order)."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pts(rng, n, lo, hi):
    return [rng.uniform(lo, hi, n).astype(np.float32) for _ in range(3)]


@pytest.mark.parametrize("periodic", [0, 1])
@pytest.mark.parametrize("k", [1, 32, 48, 100])
def test_knn_exact(gpu, periodic, k):
    rng = np.random.default_rng(10 * k + periodic)
    x, y, z = _pts(rng, 40000, -50, 50)
    q = _pts(rng, 5000, -50, 50)
    L = 100.0 if periodic else 0.0
    i1, d1 = O.knn(x, y, z, *q, k, L)
    i2, d2 = gpu.knn_search(x, y, z, *q, k, L)
    assert np.array_equal(i1, i2)
    assert np.array_equal(d1, d2)


def test_knn_lattice_ties(gpu):
    g = np.arange(-8, 8, dtype=np.float32) + 0.5
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x, y, z = (a.ravel().copy() for a in (X, Y, Z))
    for L in (16.0, 0.0):
        i1, d1 = O.knn(x, y, z, x, y, z, 32, L)
        i2, d2 = gpu.knn_search(x, y, z, x, y, z, 32, L)
        assert np.array_equal(i1, i2) and np.array_equal(d1, d2)


@pytest.mark.parametrize("n", [1, 2, 7, 8, 48, 49, 1000, 65537, 1_000_003])
def test_indexx_exact(gpu, n):
    rng = np.random.default_rng(n)
    cases = [rng.integers(0, max(2, n // 20), n).astype(np.float32),
             rng.standard_normal(n).astype(np.float32),
             np.full(n, 3.0, np.float32),
             np.arange(n, dtype=np.float32),
             np.arange(n, dtype=np.float32)[::-1].copy()]
    for a in cases:
        assert np.array_equal(gpu.indexx(a), O.indexx(a))


@pytest.fixture(scope="module")
def p2g_pair(gpu, mock1):
    res = {}
    for vel, dens in ((1, 1), (0, 0), (0, 1), (1, 0)):
        p = Params(nx=64, periodic=1, lado0=100.0, flag_vel_interp=vel, flag_dens_interp=dens)
        o = O.particles_to_grid(p, *(mock1[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
        g = gpu.particles_to_grid(p, mock1)
        res[(vel, dens)] = (o, g)
    return res


def test_sph_fields_exact(p2g_pair):
    o, g = p2g_pair[(1, 1)]
    for k in ("part_dens", "hpart", "u2", "u3", "u4", "u_mass"):
        assert np.array_equal(o[k], g[k]), k


def _rel_close(a, b, tol):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    scale = np.abs(a) + np.mean(np.abs(a))
    return np.all(np.abs(a - b) <= tol * scale)


@pytest.mark.parametrize("mode", [(0, 0), (0, 1), (1, 0)])
def test_tsc_and_mixed_modes(p2g_pair, mode):
    # TSC sums in particle order (the reference's serial loop order; its OpenMP
    # atomics leave the order open): bit-exact
    o, g = p2g_pair[mode]
    for k in ("u_mass", "u2", "u3", "u4"):
        assert np.array_equal(o[k], g[k]), k
    if mode[1] == 1:
        assert np.array_equal(o["hpart"], g["hpart"])


@pytest.fixture(scope="module")
def fields_pair(gpu, oracle_mock1):
    res = {}
    for per in (1, 0):
        p = Params(nx=64, periodic=per, lado0=100.0)
        grid = oracle_mock1[per]["grid"]
        o = O.fields(p, grid["u_mass"], grid["u2"], grid["u3"], grid["u4"])
        g = gpu.fields(p, grid["u_mass"], grid["u2"], grid["u3"], grid["u4"])
        res[per] = (p, o, g)
    return res


def test_fields_exact(fields_pair):
    for per, (p, o, g) in fields_pair.items():
        assert np.array_equal(o[0], g[0]) and np.array_equal(o[1], g[1]) and o[2] == g[2]


def test_flags_exact(gpu, fields_pair):
    for per, (p, o, g) in fields_pair.items():
        vo = O.voidfind(p, o[0], o[1])
        fl = gpu.mark_all(p, o[0], o[1])
        assert np.array_equal(vo["flags"], fl)


def test_voidfind_exact(gpu, fields_pair):
    for per, (p, o, g) in fields_pair.items():
        vo = O.voidfind(p, o[0], o[1])
        cubes, nv = gpu.voidfind(p, o[0], o[1])
        assert nv == vo["nvoid"]
        for k in cubes:
            assert np.array_equal(cubes[k], vo["cubes"][k]), k


def test_merge_post_parity(gpu, fields_pair):
    for per, (p, o, g) in fields_pair.items():
        vo = O.voidfind(p, o[0], o[1])
        co = O.merge_post(p, vo["nvoid"], vo["cubes"], o[0], o[2])
        cg = gpu.merge_post(p, vo["nvoid"], vo["cubes"], o[0], o[2])
        # every column bit-exact: the REAL*4 inertia, UMEAN and MTOT sums run in
        # the reference's serial K, J, I order per void on the GPU too
        for k in ("indice", "uvoid", "ncellv", "marca", "volnew", "req", "xc", "yc", "zc", "gxc", "gyc", "gzc",
                  "eps", "ip", "umean", "mtot"):
            assert np.array_equal(co[k], cg[k]), k
        assert (co["nvoid2"], co["nvoidt"], co["volt_clean"]) == (cg["nvoid2"], cg["nvoidt"], cg["volt_clean"])


def test_run_level_matches_oracle(gpu, mock1, oracle_mock1):
    for per in (1, 0):
        p = Params(nx=64, periodic=per, lado0=100.0)
        r = gpu.run_level(p, mock1, capacity=100000, want_marca=True)
        o = oracle_mock1[per]
        assert r["nvoid"] == o["vf"]["nvoid"]
        for k in r["cubes"]:
            assert np.array_equal(r["cubes"][k], o["vf"]["cubes"][k]), k
        assert r["meandens"] == o["meandens"]
        for k in ("indice", "uvoid", "ncellv", "marca", "volnew", "req", "gxc", "gyc", "gzc", "eps", "ip",
                  "umean", "mtot"):
            assert np.array_equal(r["cat"][k], o["cat"][k]), k
        assert r["cat"]["nvoidt"] == o["cat"]["nvoidt"] and r["cat"]["nvoidt"] > 0


def test_run_level_deterministic(gpu, mock1):
    p = Params(nx=64, periodic=1, lado0=100.0)
    a = gpu.run_level(p, mock1, capacity=100000)
    b = gpu.run_level(p, mock1, capacity=100000)
    for k in a["cat"]:
        assert np.array_equal(np.asarray(a["cat"][k]), np.asarray(b["cat"][k])), k


def test_run_level_into_caller_buffers(gpu, mock1):
    """Reused caller-owned arrays (level_buffers) give the same catalogue, also
    when a larger previous result is left in them."""
    p = Params(nx=64, periodic=1, lado0=100.0)
    want = gpu.run_level(p, mock1, capacity=100000, want_marca=True)
    bufs = gpu.level_buffers(p, capacity=100000, want_marca=True)
    for a in list(bufs[0].arr.values()) + list(bufs[1].arr.values()):
        a[:] = 7
    for _ in range(2):
        got = gpu.run_level(p, mock1, bufs=bufs, want_marca=True)
        assert got["nvoid"] == want["nvoid"]
        for k in want["cubes"]:
            assert np.array_equal(got["cubes"][k], want["cubes"][k]), k
        for k in want["cat"]:
            assert np.array_equal(np.asarray(got["cat"][k]), np.asarray(want["cat"][k])), k


def test_catalogue_independent_of_binning(gpu, mock1, monkeypatch):
    """The kNN is exact for any bin size and for any starting radius (plain,
    learned, density estimate), so these knobs change timing only."""
    p = Params(nx=64, periodic=1, lado0=100.0)
    base = gpu.run_level(p, mock1, capacity=100000)
    from avism_b200 import proposal
    gpu.proposal_load(proposal.load_weights())
    variants = [("0.5", 0), ("4", 0), ("2", 1), ("1", 1), ("2", 2)]
    for occ, learned in variants:
        monkeypatch.setenv("AVISM_TUNE_OCC", occ)
        q = Params(nx=64, periodic=1, lado0=100.0, learned=learned)
        r = gpu.run_level(q, mock1, capacity=100000)
        assert r["nvoid"] == base["nvoid"]
        for k in base["cubes"]:
            assert np.array_equal(r["cubes"][k], base["cubes"][k]), (occ, learned, k)
        for k in base["cat"]:
            assert np.array_equal(np.asarray(r["cat"][k]), np.asarray(base["cat"][k])), (occ, learned, k)


def test_out_of_box_is_an_error(gpu, mock_small):
    from avism_b200.avism import AvismError
    parts = {k: np.array(v, copy=True) for k, v in mock_small.items() if isinstance(v, np.ndarray)}
    parts["x"][5] = 40.0                       # box is [-32, 32]
    p = Params(nx=32, periodic=1, lado0=64.0)
    with pytest.raises(AvismError) as e:
        gpu.run_level(p, parts, capacity=10000)
    assert e.value.code == 5


def test_nvoid_max_matches_reference_stop(gpu, fields_pair):
    """'NVOID > NVOID_MAX!! Increase NVOID_MAX' fires exactly when the oracle's does."""
    from avism_b200.avism import AvismError
    p0, o, _ = fields_pair[1]
    nv = O.voidfind(p0, o[0], o[1])["nvoid"]
    for cap in (nv - 1, nv, nv + 1):
        p = Params(nx=64, periodic=1, lado0=100.0, nvoid_max=cap)
        try:
            O.voidfind(p, o[0], o[1])
            ref_err = None
        except O.OracleError as e:
            ref_err = str(e)
        if ref_err is None:
            cubes, n = gpu.voidfind(p, o[0], o[1], capacity=cap)
            assert n == nv
        else:
            assert "4" in ref_err
            with pytest.raises(AvismError) as e:
                gpu.voidfind(p, o[0], o[1], capacity=cap)
            assert e.value.code == 4


def test_next_level_parent_map(gpu, mock1, oracle_mock1):
    """a26: the next level's MARCAP2 and REQP from the level-0 catalogue."""
    for per in (1, 0):
        p = Params(nx=64, periodic=per, lado0=100.0)
        o = oracle_mock1[per]
        nv = o["vf"]["nvoid"]
        mg, rg = gpu.next_level(p, nv, o["cat"]["marca"], o["cat"]["uvoid"], o["cat"]["req"])
        mo, ro = O.next_level(p, nv, o["cat"]["marca"], o["cat"]["uvoid"], o["cat"]["req"])
        assert np.array_equal(mg, mo) and np.array_equal(rg, ro)


def test_voids_in_voids_two_levels(gpu):
    """Level 0 at 32^3, then level 1 at 64^3 inside the level-0 voids, against
    the oracle's same sequence (cubes and catalogue ids bit-exact)."""
    from avism_b200 import synth
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 17, box=64.0, nsph=4, rmin=7.0, rmax=11.0, seed=77))
    p0 = Params(nx=32, periodic=1, lado0=64.0, rmin=2.0, rmin_sub=2.0)
    o0 = O.run_level(p0, parts)
    g0 = gpu.run_level(p0, parts, capacity=100000, want_marca=True)
    assert np.array_equal(g0["cat"]["marca"], o0["cat"]["marca"])
    nv = o0["vf"]["nvoid"]
    mp, rq = O.next_level(p0, nv, o0["cat"]["marca"], o0["cat"]["uvoid"], o0["cat"]["req"])
    assert np.any(mp > 0)
    p1 = Params(nx=64, periodic=1, lado0=64.0, rmin=2.0, rmin_sub=2.0, level=1)
    o1 = O.run_sublevel(p1, parts, mp, rq)
    g1 = gpu.run_sublevel(p1, parts, mp, rq, capacity=100000, want_marca=True)
    assert g1["nvoid"] == o1["vf"]["nvoid"]
    for k in g1["cubes"]:
        assert np.array_equal(g1["cubes"][k], o1["vf"]["cubes"][k]), k
    for k in ("indice", "uvoid", "ncellv", "marca", "volnew", "req", "gxc", "gyc", "gzc"):
        assert np.array_equal(g1["cat"][k], o1["cat"][k]), k
    # every level-1 cube grows inside a level-0 void
    father = np.asarray(g1["cubes"]["father"])
    assert np.all(father > 0)


@pytest.mark.parametrize("case", ["straddling", "overlapping"])
def test_known_answer_fields_match_oracle(gpu, case):
    """The oracle's known-answer voids (a void across the periodic boundary, two
    overlapping holes merged into one) give the same catalogue on the GPU."""
    import test_oracle_pins as K
    L = 64.0
    if case == "straddling":
        parts = K._void_field(2 ** 16, L, [(np.array([L / 2 - 2.0, 5.0, -7.0]), 12.0)], 0.1, 0.5, seed=21)
    else:
        parts = K._void_field(2 ** 16, L, [(np.array([-5.0, 0.0, 0.0]), 9.0), (np.array([5.0, 0.0, 0.0]), 9.0)],
                              0.1, 0.5, seed=22)
    p = Params(nx=32, lado0=L, periodic=1, rmin=2.0)
    o = O.run_level(p, parts)
    g = gpu.run_level(p, parts, capacity=100000)
    assert g["nvoid"] == o["vf"]["nvoid"]
    for k in ("indice", "uvoid", "ncellv"):
        assert np.array_equal(np.asarray(g["cat"][k]), np.asarray(o["cat"][k])), k
    for k in ("volnew", "gxc", "gyc", "gzc"):
        assert np.array_equal(np.asarray(g["cat"][k]), np.asarray(o["cat"][k])), k
    assert g["cat"]["nvoidt"] == o["cat"]["nvoidt"]


def test_survey_mask_paths(gpu, mock1):
    """SMASK (survey mode's observed-cell mask): no SPH interpolation in masked
    cells, and no flag, centre or growth through them -- as in the oracle."""
    p = Params(nx=64, periodic=1, lado0=100.0)
    g, radx = O.grid_setup(p)
    rad = radx.astype(np.float64)

    def sphere_mask(lo, n):                       # observed: within 35 cMpc of the origin
        i = np.arange(n ** 3)
        c = [rad[(i // n ** a) % n + lo - g.rad_lo] for a in range(3)]
        return ((c[0] ** 2 + c[1] ** 2 + c[2] ** 2) < 35.0 ** 2).astype(np.int8)

    smask = sphere_mask(1, g.nx)
    args = [mock1[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
    o = O.particles_to_grid(p, *args, smask=smask)
    gg = gpu.particles_to_grid(p, mock1, smask=smask)
    for k in ("part_dens", "hpart", "u2", "u3", "u4", "u_mass"):
        assert np.array_equal(o[k], gg[k]), k
    assert np.all(o["u2"][smask == 0] == 0.0)
    smask_ext = sphere_mask(g.low1, g.ne)
    u1, dv, _ = O.fields(p, o["u_mass"], o["u2"], o["u3"], o["u4"])
    vo = O.voidfind(p, u1, dv, smask_ext=smask_ext)
    assert np.array_equal(vo["flags"], gpu.mark_all(p, u1, dv, smask_ext=smask_ext))
    cubes, nv = gpu.voidfind(p, u1, dv, smask_ext=smask_ext)
    assert nv == vo["nvoid"] > 0
    for k in cubes:
        assert np.array_equal(cubes[k], vo["cubes"][k]), k


@pytest.mark.parametrize("k,periodic", [(16, 1), (48, 1), (48, 0), (100, 1)])
def test_sph_fields_other_k(gpu, mock_small, k, periodic):
    """The SPH fields for k other than 32 (the 64- and 128-wide warp kNN
    instantiations and the counting select), periodic and not."""
    p = Params(nx=32, periodic=periodic, lado0=64.0, kneighbours=k)
    o = O.particles_to_grid(p, *(mock_small[q] for q in ("x", "y", "z", "vx", "vy", "vz", "m")))
    g = gpu.particles_to_grid(p, mock_small)
    for key in ("part_dens", "hpart", "u2", "u3", "u4", "u_mass"):
        assert np.array_equal(o[key], g[key]), key
