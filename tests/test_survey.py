"""Survey mode on the CPU (src/avism.f90:1420-1596): the oracle's D/(alpha R)
contrast against a numpy restatement, and the survey inputs read through the
library's file readers (mask.dat, rands.dat) into a whole survey level."""
import numpy as np
import pytest

from avism_b200 import synth
from avism_b200._abi import Params, UM
from oracle import oracle as O

GEO = dict(box=150.0, rmax=75.0, half_angle_deg=60.0)


@pytest.fixture(scope="module")
def survey():
    c = synth.weighted_cone(ng=64, rsel=50.0, n_target=20000, seed=1005, **GEO)
    parts = synth.to_reader_units(c)
    rands = synth.cone_randoms(60000, c["pixel_mask"], rsel=50.0, seed=2005, **GEO)
    rands["w"] = (rands["w"] / UM).astype(np.float32)
    smask = synth.cone_mask(64, c["pixel_mask"], **GEO)
    return parts, rands, smask


def test_contrast_matches_numpy(survey):
    parts, rands, smask = survey
    p = Params(nx=64, periodic=0, lado0=150.0, kneighbours=16, flag_vel_interp=0, flag_dens_interp=0,
               no_velocities=1)
    u1, dv, md, ur = O.survey_fields(p, {k: v for k, v in parts.items() if k not in ("vx", "vy", "vz")}, rands,
                                     smask)
    g, _ = O.grid_setup(p)
    # the tracers' density in rho_B units times ROTE, then D/(alpha R) in REAL*8
    o = O.particles_to_grid(p, *(parts.get(k) for k in ("x", "y", "z", "vx", "vy", "vz", "m")), smask=smask)
    dx = np.float32(g.dx)
    vol = np.float32(dx * dx * dx) * np.float32(np.float32(g.rete * g.rete) * g.rete)
    d = ((o["u_mass"] / vol) / np.float32(g.rote)) * np.float32(g.rote)
    obs = smask != 0
    alpha = d[obs].astype(np.float64).sum() / ur[obs].astype(np.float64).sum()
    ratio = np.where(ur > 0, d.astype(np.float64) / (alpha * ur.astype(np.float64)), np.float64(np.float32(1e-4)))
    ratio = np.clip(ratio, np.float64(np.float32(1e-4)), 1000.0).astype(np.float32)
    pos = smask > 0
    mean = np.float32(ratio[pos].astype(np.float64).mean())
    want = np.where(pos, ratio / mean, np.where(obs, ratio, d)).astype(np.float32)
    got = u1.reshape(g.ne, g.ne, g.ne)                     # non-periodic: ext == inner
    assert np.allclose(got.ravel(), want, rtol=2e-7, atol=0)
    assert abs(got.ravel()[pos].astype(np.float64).mean() - 1.0) < 1e-6
    # MEANDENS = ROTE * UM / UL^3 (background density), not the tracers' mean
    assert md == np.float32(g.rote) * np.float32(np.float32(UM) / np.float32(np.float32(10.98) ** 3))
    # linear-theory divergence of the contrast
    coef = np.float32(np.float32(np.float32(0.31) ** np.float32(0.6)) * np.float32(g.rete)) * np.float32(g.hte)
    assert np.allclose(dv, -coef * (u1 - np.float32(1)), rtol=1e-6, atol=1e-12)


def test_survey_inputs_from_files(tmp_path, survey):
    """mask.dat and rands.dat written in the reference's layouts, read with the
    library's readers, give the same survey level as the arrays themselves."""
    from avism_b200.avism import read_mask_file, read_randoms_file
    parts, rands, smask = survey
    mp = tmp_path / "mask.dat"
    with open(mp, "wb") as f:
        f.write(np.int32(64).tobytes() + np.array([0.0, 75.0, 150.0], np.float32).tobytes() + smask.tobytes())
    rp = tmp_path / "rands.dat"
    w_msun = (rands["w"] * np.float32(UM)).astype(np.float32)
    with open(rp, "wb") as f:
        for rec in [np.int32(len(rands["x"])).tobytes()] + [a.tobytes() for a in (rands["x"], rands["y"],
                                                                                   rands["z"], w_msun)]:
            f.write(np.uint32(len(rec)).tobytes() + rec + np.uint32(len(rec)).tobytes())
    sm2, _ = read_mask_file(mp, 64, 64)
    rr = read_randoms_file(rp)
    assert np.array_equal(sm2, smask)
    rr["w"] = (rr["w"] / UM).astype(np.float32)
    p = Params(nx=64, periodic=0, lado0=150.0, kneighbours=16, flag_vel_interp=0, flag_dens_interp=0,
               no_velocities=1, rmin=3.0)
    novel = {k: v for k, v in parts.items() if k not in ("vx", "vy", "vz")}
    a = O.run_level_survey(p, novel, rands, smask)
    b = O.run_level_survey(p, novel, rr, sm2)
    assert a["vf"]["nvoid"] == b["vf"]["nvoid"] > 0
    assert np.array_equal(a["cat"]["marca"], b["cat"]["marca"])
