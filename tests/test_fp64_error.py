"""Error of the REAL*4 particle-to-grid path against the same method in FP64.

The GPU's SPH fields equal the oracle's bit for bit (test_gpu_parity), so the
oracle's error against oracle/fp64.py is the GPU's error too.  Bounds (32^3
mock, 2^15 particles; the 64^3 / 2^18 figures are of the same size):
part_dens, hpart and u_mass within 1e-5 relative everywhere; velocities within
1e-5 of |v| + mean |v| at the 99th percentile and 1e-4 at most."""
import numpy as np
import pytest

from avism_b200 import synth
from avism_b200._abi import Params
from oracle import oracle as O
from oracle.fp64 import particles_to_grid_fp64


@pytest.fixture(scope="module")
def pair():
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=50.0, seed=1001))
    p = Params(nx=32, periodic=1, lado0=50.0)
    args = [parts[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
    return O.particles_to_grid(p, *args), particles_to_grid_fp64(p, *args)


def _rel(a, b, add_mean=False):
    a = a.astype(np.float64)
    scale = np.abs(b) + (np.mean(np.abs(b)) if add_mean else 0.0)
    return np.abs(a - b) / np.where(scale > 0, scale, 1.0)


@pytest.mark.parametrize("field", ["part_dens", "hpart", "u_mass"])
def test_scalar_fields_within_1e5_of_fp64(pair, field):
    f32, f64 = pair
    assert np.all(f64[field] >= 0)
    assert np.max(_rel(f32[field], f64[field])) < 1e-5


@pytest.mark.parametrize("field", ["u2", "u3", "u4"])
def test_velocities_close_to_fp64(pair, field):
    f32, f64 = pair
    r = _rel(f32[field], f64[field], add_mean=True)
    assert np.quantile(r, 0.99) < 1e-5
    assert np.max(r) < 1e-4


def test_fp64_restatement_conserves_mass(pair):
    _, f64 = pair
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=50.0, seed=1001))
    # DDENS does not wrap: only mass whose support leaves the grid is lost
    total = np.sum(np.asarray(parts["m"], np.float64))
    assert 0.9 * total < np.sum(f64["u_mass"]) <= total * (1 + 1e-12)


@pytest.mark.parametrize("periodic", [1, 0])
def test_tsc_fields_close_to_fp64(periodic):
    """TSC density and velocity (the GPU's are within 1e-5 of the oracle's)."""
    from oracle.fp64 import tsc_fp64
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=50.0, seed=1001))
    p = Params(nx=32, periodic=periodic, lado0=50.0, flag_vel_interp=0, flag_dens_interp=0)
    args = [parts[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
    f32, f64 = O.particles_to_grid(p, *args), tsc_fp64(p, *args)
    r = _rel(f32["u_mass"], f64["u_mass"])
    assert np.quantile(r, 0.99) < 1e-6 and np.max(r) < 1e-4
    for k in ("u2", "u3", "u4"):
        assert np.max(_rel(f32[k], f64[k], add_mean=True)) < 1e-5, k


def test_fp64_restatement_against_brute_force():
    """Pin oracle/fp64.py itself: PPART_DENS, one cell's VVEL and one particle's
    DDENS support recomputed with plain loops over all particles / cells."""
    rng = np.random.default_rng(3)
    L, nx, K, n = 16.0, 8, 8, 600
    x, y, z = (rng.uniform(-L / 2, L / 2, n).astype(np.float32) for _ in range(3))
    vx, vy, vz = (rng.normal(0, 100, n).astype(np.float32) for _ in range(3))
    m = np.full(n, 2.0, np.float32)
    p = Params(nx=nx, periodic=1, lado0=L, kneighbours=K)
    f = particles_to_grid_fp64(p, x, y, z, vx, vy, vz, m)
    P = np.stack([x, y, z], 1).astype(np.float64)

    def dist(a, b):
        d = np.abs(a - b)
        d = np.minimum(d, L - d)
        return np.sqrt((d ** 2).sum(-1))

    # PPART_DENS of particle 5: K nearest (itself included), mass over the ball of the K-th distance
    d5 = np.sort(dist(P, P[5]))
    assert np.isclose(f["part_dens"][5], 2.0 * K / (4.0 / 3.0 * np.pi * d5[K - 1] ** 3), rtol=1e-12)
    # VVEL of cell (3, 4, 5): M4 weights over its K nearest, m / rho_p
    g, radx = O.grid_setup(p)
    rad = radx.astype(np.float64)
    q = np.array([rad[3 - g.rad_lo], rad[4 - g.rad_lo], rad[5 - g.rad_lo]])
    dq = dist(P, q)
    nn = np.argsort(dq, kind="stable")[:K]
    h = dq[nn].max()
    assert h > float(g.dx)                                  # the kNN branch, not the ball
    qq = dq[nn] / (h / 2)
    w = np.where(qq <= 1, 1 - 1.5 * qq ** 2 * (1 - 0.5 * qq), np.where(qq <= 2, 0.25 * (2 - qq) ** 3, 0))
    w = w * 2.0 / f["part_dens"][nn]
    c = (3 - 1) + nx * ((4 - 1) + nx * (5 - 1))
    assert np.isclose(f["u2"][c], (w * vx[nn]).sum() / w.sum(), rtol=1e-12)
    # DDENS: the grid total is the mass of the particles whose supports stay in the grid
    assert 0.5 * m.sum() < f["u_mass"].sum() <= m.sum() * (1 + 1e-12)


def test_gaussian_kernel_within_bounds_of_fp64():
    """KERNEL_MODE = 2 (Gaussian, src/particles.f90:535-538, 955-956): the REAL*4
    fields against FP64 -- scalar fields within 1e-5 relative, velocities within
    1e-5 of |v| + mean |v| at the 99th percentile.  The GPU calls CUDA's expf,
    the oracle the host's: their fields agree to the same 1e-5 (GPU test)."""
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 14, box=50.0, seed=1002))
    p = Params(nx=24, periodic=1, lado0=50.0, kernel_mode=2)
    args = [parts[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
    f32, f64 = O.particles_to_grid(p, *args), particles_to_grid_fp64(p, *args)
    m4 = O.particles_to_grid(Params(nx=24, periodic=1, lado0=50.0), *args)
    assert not np.array_equal(f32["u_mass"], m4["u_mass"])          # the kernel changed the fields
    assert np.array_equal(f32["hpart"], m4["hpart"])                 # but not h
    for k in ("part_dens", "hpart", "u_mass"):
        assert np.max(_rel(f32[k], f64[k])) < 1e-5, k
    for k in ("u2", "u3", "u4"):
        r = _rel(f32[k], f64[k], add_mean=True)
        assert np.quantile(r, 0.99) < 1e-5 and np.max(r) < 1e-4, k
