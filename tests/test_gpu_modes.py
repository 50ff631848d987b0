"""GPU parity of the reference's other particle modes:
  * no velocities (FLAG_VEL_AVAILABLE = 0, READ_BINARY_PART_2 input): density
    only, H_DISTANCE + FILL_H_ZEROS + DDENS (or TSC), and the linear-theory
    divergence -Omega_m^0.6 a H (rho/rho_mean - 1) (src/avism.f90:1259-1306,
    1647-1650) -- bit-exact through the whole level;
  * the Gaussian SPH kernel (KERNEL_MODE = 2, src/particles.f90:535-538,
    955-956) -- the GPU's expf against the host's: within 1e-5."""
import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _novel(parts):
    return {k: v for k, v in parts.items() if k not in ("vx", "vy", "vz")}


@pytest.mark.parametrize("dens,periodic", [(1, 1), (0, 1), (1, 0)])
def test_no_velocity_level_exact(gpu, mock_small, dens, periodic):
    parts = _novel(mock_small)
    p = Params(nx=32, periodic=periodic, lado0=64.0, flag_dens_interp=dens, no_velocities=1, rmin=2.0)
    o = O.run_level(p, parts)
    g = gpu.particles_to_grid(p, parts)
    for k in ("u_mass", "hpart", "u2"):
        assert np.array_equal(o["grid"][k], g[k]), k
    assert not np.any(g["u2"])
    u1, dv, md = gpu.fields(p, g["u_mass"], None, None, None)
    assert np.array_equal(u1, o["u1co"]) and np.array_equal(dv, o["diverco"]) and md == o["meandens"]
    # the linear-theory divergence: -(coef * (delta + 1 - 1)) with coef = Omega_m^0.6 a H in REAL*4
    gg, _ = O.grid_setup(p)
    coef = np.float32(np.float32(np.float32(p.omega0) ** np.float32(0.6)) * np.float32(gg.rete)) * np.float32(gg.hte)
    assert np.allclose(dv, -coef * (u1 - np.float32(1.0)), rtol=1e-6, atol=0)
    r = gpu.run_level(p, parts, capacity=100000)
    assert r["nvoid"] == o["vf"]["nvoid"] > 0
    for k in r["cubes"]:
        assert np.array_equal(r["cubes"][k], o["vf"]["cubes"][k]), k
    for k in ("indice", "uvoid", "ncellv", "volnew", "req", "gxc", "gyc", "gzc"):
        assert np.array_equal(np.asarray(r["cat"][k]), np.asarray(o["cat"][k])), k


def _close(a, b, tol, add_mean):
    a, b = a.astype(np.float64), b.astype(np.float64)
    scale = np.abs(b) + (np.mean(np.abs(b)) if add_mean else 0.0)
    return np.max(np.abs(a - b) / np.where(scale > 0, scale, 1.0)) <= tol


@pytest.mark.parametrize("vel,dens", [(1, 1), (0, 1)])
def test_gaussian_kernel_within_1e5(gpu, mock_small, vel, dens):
    p = Params(nx=32, periodic=1, lado0=64.0, kernel_mode=2, flag_vel_interp=vel, flag_dens_interp=dens)
    o = O.particles_to_grid(p, *(mock_small[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
    g = gpu.particles_to_grid(p, mock_small)
    # no kernel in the neighbour distances and densities: bit-exact
    for k in ("hpart", "part_dens"):
        assert np.array_equal(o[k], g[k]), k
    assert _close(g["u_mass"], o["u_mass"], 1e-5, False)
    if vel == 1:
        for k in ("u2", "u3", "u4"):
            assert _close(g[k], o[k], 1e-5, True), k
    m4 = gpu.particles_to_grid(Params(nx=32, periodic=1, lado0=64.0, flag_vel_interp=vel,
                                      flag_dens_interp=dens), mock_small)
    assert not np.array_equal(m4["u_mass"], g["u_mass"])
