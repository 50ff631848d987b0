"""GPU parity of survey mode (FLAG_SURVEY = 1, src/avism.f90:1420-1596) against
the oracle: a weighted tracer cone with radial selection and an angular mask,
its randoms and the mask grid; the randoms' SPH kNN with KNEIGHBOURS2 =
MIN(8*KNEIGHBOURS, 256) neighbours, the D/(alpha R) contrast, the divergence and
the whole level, bit for bit."""
import numpy as np
import pytest

from avism_b200 import synth
from avism_b200._abi import Params, UM
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GEO = dict(box=150.0, rmax=75.0, half_angle_deg=60.0)


@pytest.fixture(scope="module")
def survey():
    c = synth.weighted_cone(ng=64, rsel=50.0, n_target=20000, seed=1005, **GEO)
    parts = synth.to_reader_units(c)
    rands = synth.cone_randoms(60000, c["pixel_mask"], rsel=50.0, seed=2005, **GEO)
    rands["w"] = (rands["w"] / UM).astype(np.float32)
    smask = synth.cone_mask(64, c["pixel_mask"], **GEO)
    return parts, rands, smask


MODES = [(1, 1, 0, 16), (0, 1, 1, 16), (0, 0, 1, 16), (0, 1, 1, 32)]


@pytest.mark.parametrize("vel,dens,novel,k", MODES)
def test_survey_fields_exact(gpu, survey, vel, dens, novel, k):
    parts, rands, smask = survey
    if novel:
        parts = {q: v for q, v in parts.items() if q not in ("vx", "vy", "vz")}
    p = Params(nx=64, periodic=0, lado0=150.0, kneighbours=k, flag_vel_interp=vel, flag_dens_interp=dens,
               no_velocities=novel, rmin=3.0)
    o = O.survey_fields(p, parts, rands, smask)
    g = gpu.survey_fields(p, parts, rands, smask)
    assert np.array_equal(o[3], g[3])                  # the randoms' grid
    assert np.array_equal(o[0], g[0])                  # U1CO = D/(alpha R)
    assert np.array_equal(o[1], g[1])                  # DIVERCO
    assert o[2] == g[2]


@pytest.mark.parametrize("vel,dens,novel,k", MODES[:3])
def test_survey_level_exact(gpu, survey, vel, dens, novel, k):
    parts, rands, smask = survey
    if novel:
        parts = {q: v for q, v in parts.items() if q not in ("vx", "vy", "vz")}
    p = Params(nx=64, periodic=0, lado0=150.0, kneighbours=k, flag_vel_interp=vel, flag_dens_interp=dens,
               no_velocities=novel, rmin=3.0)
    o = O.run_level_survey(p, parts, rands, smask)
    r = gpu.run_level_survey(p, parts, rands, smask, capacity=200000, want_marca=True)
    assert r["nvoid"] == o["vf"]["nvoid"] > 0
    for q in r["cubes"]:
        assert np.array_equal(r["cubes"][q], o["vf"]["cubes"][q]), q
    for q in ("indice", "uvoid", "ncellv", "marca", "volnew", "req", "xc", "yc", "zc", "gxc", "gyc", "gzc", "eps",
              "ip", "umean", "mtot"):
        assert np.array_equal(np.asarray(r["cat"][q]), np.asarray(o["cat"][q])), q
    assert r["cat"]["nvoidt"] == o["cat"]["nvoidt"] and r["meandens"] == o["meandens"]
