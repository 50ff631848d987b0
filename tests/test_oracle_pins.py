"""Pins of the CPU oracle (no GPU needed).

The reference ships no golden vectors and cannot be compiled here, so the oracle
is pinned against independent Python restatements of the reference routines and
against analytic known-answer cases."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O


# ---- INDEXX: independent Python restatement of src/num.f90:2-84 -------------
def nr_indexx_py(arr):
    n = len(arr)
    a = [None] + [float(v) for v in arr]           # 1-based
    indx = list(range(0, n + 1))
    M, stack, l, ir = 7, [], 1, n
    while True:
        if ir - l < M:
            for j in range(l + 1, ir + 1):
                t = indx[j]
                v = a[t]
                i = j - 1
                while i >= 1:
                    if a[indx[i]] <= v:
                        break
                    indx[i + 1] = indx[i]
                    i -= 1
                indx[i + 1] = t
            if not stack:
                return np.array(indx[1:], np.int32)
            ir = stack.pop()
            l = stack.pop()
        else:
            k = (l + ir) // 2
            indx[k], indx[l + 1] = indx[l + 1], indx[k]
            if a[indx[l + 1]] > a[indx[ir]]:
                indx[l + 1], indx[ir] = indx[ir], indx[l + 1]
            if a[indx[l]] > a[indx[ir]]:
                indx[l], indx[ir] = indx[ir], indx[l]
            if a[indx[l + 1]] > a[indx[l]]:
                indx[l + 1], indx[l] = indx[l], indx[l + 1]
            i, j = l + 1, ir
            t = indx[l]
            v = a[t]
            while True:
                i += 1
                while a[indx[i]] < v:
                    i += 1
                j -= 1
                while a[indx[j]] > v:
                    j -= 1
                if j < i:
                    break
                indx[i], indx[j] = indx[j], indx[i]
            indx[l] = indx[j]
            indx[j] = t
            if ir - i + 1 >= j - l:
                stack += [i, ir]
                ir = j - 1
            else:
                stack += [l, j - 1]
                l = i


@pytest.mark.parametrize("n", [1, 2, 6, 7, 8, 9, 31, 100, 1000, 4097])
def test_indexx_matches_python_restatement(n):
    rng = np.random.default_rng(n)
    for arr in (rng.integers(0, max(2, n // 7), n).astype(np.float32),
                rng.standard_normal(n).astype(np.float32),
                np.zeros(n, np.float32), np.arange(n, dtype=np.float32)[::-1].copy()):
        got = O.indexx(arr)
        assert np.array_equal(got, nr_indexx_py(arr))
        assert np.all(np.diff(arr[got - 1]) >= 0)


def test_indexx_is_not_stable():
    # equal keys leave INDEXX in a specific, non-stable order: ties matter
    arr = np.array([1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0], np.float32)
    got = O.indexx(arr)
    assert np.array_equal(got, nr_indexx_py(arr))
    assert not np.array_equal(got, np.argsort(arr, kind="stable") + 1)


# ---- kNN: brute force with the reference distance, ties by index -------------
def brute_knn(x, y, z, q, k, L):
    px, py, pz = (np.asarray(v, np.float32) for v in (x, y, z))
    out_i, out_d = [], []
    for qq in zip(*q):
        d = []
        for p_, q_ in ((px, qq[0]), (py, qq[1]), (pz, qq[2])):
            dd = (p_ - np.float32(q_)).astype(np.float32)
            if L > 0:
                a = np.abs(dd)
                dd = np.minimum(a, np.float32(L) - a)
            d.append((dd * dd).astype(np.float32))
        d2 = ((d[0] + d[1]).astype(np.float32) + d[2]).astype(np.float32)
        order = np.lexsort((np.arange(len(d2)), d2))[:k]
        out_i.append(order + 1)
        out_d.append(np.sqrt(d2[order]).astype(np.float32))
    return np.array(out_i), np.array(out_d)


@pytest.mark.parametrize("periodic", [0, 1])
def test_knn_matches_bruteforce(periodic):
    rng = np.random.default_rng(3 + periodic)
    n = 3000
    x, y, z = (rng.uniform(-10, 10, n).astype(np.float32) for _ in range(3))
    # a lattice block adds exact distance ties
    g = np.arange(-3, 3, dtype=np.float32) + 0.5
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x, y, z = (np.concatenate([a, b.ravel()]) for a, b in ((x, X), (y, Y), (z, Z)))
    q = [rng.uniform(-10, 10, 60).astype(np.float32) for _ in range(3)]
    q = [np.concatenate([a, b.ravel()[:40]]) for a, b in zip(q, (X, Y, Z))]
    L = 20.0 if periodic else 0.0
    i1, d1 = O.knn(x, y, z, *q, 32, L)
    i2, d2 = brute_knn(x, y, z, q, 32, L)
    assert np.array_equal(i1, i2)
    assert np.array_equal(d1, d2)


# ---- grid: MALLA + PBC sizes of the benchmark configurations ------------------
@pytest.mark.parametrize("nx,L,nplus,ne", [(64, 100.0, 32, 128), (256, 250.0, 51, 358),
                                           (128, 250.0, 25, 178), (512, 500.0, 64, 640)])
def test_grid_sizes(nx, L, nplus, ne):
    g, rad = O.grid_setup(Params(nx=nx, lado0=L, periodic=1))
    assert (g.nplus, g.ne, g.low1, g.low2) == (nplus, ne, 1 - nplus, nx + nplus)
    f = np.float32
    lado = f(L) - f(L) / f(nx)
    a = -lado / f(2)
    c = (lado / f(2) - a) / f(nx - 1)
    inner = rad[1 - g.rad_lo: nx + 1 - g.rad_lo]
    assert np.array_equal(inner, (a + np.arange(nx, dtype=f) * c).astype(f))
    assert g.dx == np.float32((a + c) - a)


def test_grid_nonperiodic_has_no_ghosts():
    g, rad = O.grid_setup(Params(nx=64, lado0=100.0, periodic=0))
    assert (g.nplus, g.low1, g.low2, g.ne) == (0, 1, 64, 64)


# ---- known-answer pipeline cases ------------------------------------------------
def lattice_particles(n_side, L, vel=None):
    h = L / n_side
    g = (-L / 2 + (np.arange(n_side) + 0.25) * h).astype(np.float32)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    n = X.size
    v = np.zeros(n, np.float32)
    return dict(x=X.ravel().copy(), y=Y.ravel().copy(), z=Z.ravel().copy(), vx=v.copy(), vy=v.copy(),
                vz=v.copy(), m=np.full(n, 1e-8, np.float32))


def test_uniform_lattice_has_no_voids():
    p = Params(nx=16, lado0=32.0, periodic=1, kneighbours=16)
    r = O.run_level(p, lattice_particles(32, 32.0))
    u = r["u1co"]
    # ties of the lattice's equidistant neighbours are broken by index, so h
    # (and the local density) is not uniform; the mean and the zero flow are exact
    assert abs(float(u.astype(np.float64).mean()) - 1.0) < 1e-6
    assert np.all(r["diverco"] == 0.0)
    parts = lattice_particles(32, 32.0)
    m_grid = float(r["grid"]["u_mass"].astype(np.float64).sum())
    assert abs(m_grid / float(parts["m"].astype(np.float64).sum()) - 1.0) < 1e-6   # mass conserved
    assert r["vf"]["ncand"] == 0 and r["vf"]["nvoid"] == 0
    assert r["cat"]["nvoidt"] == 0


def test_single_tophat_void():
    from avism_b200 import synth
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 16, box=64.0, nsph=1, rmin=12.0, rmax=12.0,
                                                     contrast=0.1, sigma_v=30.0, outflow=0.5, seed=11))
    c = parts["centres"][0]
    p = Params(nx=32, lado0=64.0, periodic=1, rmin=2.0)
    r = O.run_level(p, parts)
    cat = r["cat"]
    main = np.flatnonzero(cat["uvoid"] == -1)
    assert len(main) >= 1
    big = main[np.argmax(cat["volnew"][main])]
    centre = np.array([cat["gxc"][big], cat["gyc"][big], cat["gzc"][big]])
    assert np.linalg.norm(centre - c) < 4.0          # within two cells of the planted centre
    assert 6.0 < cat["req"][big] < 16.0
    assert cat["umean"][big] < 0.5


def _void_field(n, L, holes, contrast, outflow, seed):
    """Poisson particles in a periodic box with underdense spheres (centre, radius),
    which may straddle the box boundary; radial outflow inside each sphere."""
    from avism_b200 import synth
    rng = np.random.default_rng(seed)
    x = rng.uniform(-L / 2, L / 2, (4 * n, 3))
    keep = np.ones(len(x), bool)
    vel = rng.normal(0.0, 30.0, x.shape)
    for c, r in holes:
        dv = x - np.asarray(c)
        dv -= L * np.round(dv / L)                          # minimum image
        inside = np.sqrt((dv ** 2).sum(1)) < r
        keep &= ~inside | (rng.random(len(x)) < contrast)
        vel[inside] += outflow * 100.0 * dv[inside]
    x, vel = x[keep][:n], vel[keep][:n]
    parts = dict(x=x[:, 0], y=x[:, 1], z=x[:, 2], vx=vel[:, 0], vy=vel[:, 1], vz=vel[:, 2],
                 m=np.full(len(x), synth._mean_mass(len(x), L)))
    return synth.to_reader_units({k: np.asarray(v, np.float32) for k, v in parts.items()})


def _main_voids(cat):
    main = np.flatnonzero(cat["uvoid"] == -1)
    return main, np.stack([cat["gxc"][main], cat["gyc"][main], cat["gzc"][main]], 1)


def test_void_straddling_the_periodic_boundary():
    """A void centred 2 cMpc inside the +x face wraps onto the -x side: it is
    found once, at its centre modulo the box, not as two half-voids."""
    L = 64.0
    c = np.array([L / 2 - 2.0, 5.0, -7.0])
    parts = _void_field(2 ** 16, L, [(c, 12.0)], 0.1, 0.5, seed=21)
    r = O.run_level(Params(nx=32, lado0=L, periodic=1, rmin=2.0), parts)
    main, centres = _main_voids(r["cat"])
    dv = centres - c
    dv -= L * np.round(dv / L)
    near = np.sqrt((dv ** 2).sum(1)) < 8.0
    assert near.sum() == 1, centres[near]
    big = main[near][0]
    assert np.sqrt((dv[near][0] ** 2).sum()) < 4.0
    assert 6.0 < r["cat"]["req"][big] < 16.0


def test_two_overlapping_holes_merge_into_one_void():
    """Two overlapping underdense spheres give cubes at both lobes; MERGE_VOID
    joins them into one main void that owns the other lobe's cubes."""
    L = 64.0
    a, b = np.array([-5.0, 0.0, 0.0]), np.array([5.0, 0.0, 0.0])
    parts = _void_field(2 ** 16, L, [(a, 9.0), (b, 9.0)], 0.1, 0.5, seed=22)
    r = O.run_level(Params(nx=32, lado0=L, periodic=1, rmin=2.0), parts)
    cat, cubes = r["cat"], r["vf"]["cubes"]
    main, centres = _main_voids(cat)
    near = np.sqrt((centres ** 2).sum(1)) < 12.0            # main voids around the pair
    assert near.sum() == 1, centres[near]
    owner = main[near][0] + 1                                 # 1-based void id
    # the main void owns cubes grown in both lobes
    g, _ = O.grid_setup(Params(nx=32, lado0=L, periodic=1))
    cx = g.rx1 + (np.asarray(cubes["icx"], np.float64) - 1) * g.dx
    uvoid = np.asarray(cat["uvoid"])
    owned = (uvoid == owner) | (np.arange(len(uvoid)) + 1 == owner)
    assert owned.sum() >= 2
    assert cx[owned].min() < -2.0 and cx[owned].max() > 2.0


def test_req_follows_the_fortran_promotions():
    """REQ = ((3.*VOLM)/(4.*PI))**(1./3.) (src/avism.f90:2071).  VOLM is REAL*8
    (src/avism.f90:73: 'REAL*8 :: VOLT_CLEAN, VOLM') and PI REAL*8
    (src/commondata.f90:16), so 3.*VOLM, 4.*PI and the quotient are REAL*8; the
    exponent 1./3. is a REAL*4 quotient widened for the power."""
    from avism_b200 import synth
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 16, box=64.0, nsph=8, rmin=4.0, rmax=8.0, seed=5))
    r = O.run_level(Params(nx=48, lado0=64.0, periodic=1, rmin=1.0), parts)   # dx^3 not a power of two
    cat = r["cat"]
    main = np.flatnonzero(cat["uvoid"] == -1)
    v = cat["volnew"][main].astype(np.float32)
    third = np.float64(np.float32(1.0) / np.float32(3.0))
    four_pi = 4.0 * np.arccos(-1.0)
    expect = np.power(3.0 * v.astype(np.float64) / four_pi, third).astype(np.float32)
    assert np.array_equal(cat["req"][main], expect)
    # the case is one where a REAL*4 product 3.*VOLNEW would give another REQ
    wrong = np.power((np.float32(3.0) * v).astype(np.float64) / four_pi, third).astype(np.float32)
    assert np.any(wrong != expect)
