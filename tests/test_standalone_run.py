"""The standalone iteration (avism_b200/run.py) on CPU: the C oracle stands in
for the GPU engine, so the file handling, the level loop and the hand-over
between levels (MARCAP2, REQP, NVOIDP) are checked here; the GPU engine's
levels are checked against the same oracle in test_gpu_parity."""
import os

import numpy as np

from avism_b200 import synth
from avism_b200._abi import Params
from avism_b200.run import run_iteration
from oracle import oracle as O

from test_io import _fortran_records, _read_voids_file


class OracleEngine:
    """The AvismGPU methods run_iteration calls, answered by the oracle."""

    @staticmethod
    def _res(r):
        return dict(cubes=r["vf"]["cubes"], nvoid=r["vf"]["nvoid"], cat=r["cat"], meandens=r["meandens"])

    def run_level(self, p, parts, want_marca=False):
        return self._res(O.run_level(p, parts))

    def run_sublevel(self, p, parts, marcap, reqp, want_marca=False):
        return self._res(O.run_sublevel(p, parts, marcap, reqp))

    def next_level(self, p, nvoid, marca, uvoid, req):
        return O.next_level(p, nvoid, marca, uvoid, req)

    def particles_to_grid(self, p, parts):
        return O.particles_to_grid(p, *(parts[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")))

    def fields(self, p, *grids):
        return O.fields(p, *grids)


def test_two_level_iteration_files(tmp_path):
    raw = synth.mock_spheres(n=2 ** 16, box=64.0, nsph=4, rmin=7.0, rmax=11.0, seed=77)
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")
    n = len(raw["x"])
    path = tmp_path / "bin_file_part00001"
    _fortran_records(path, [np.int64(n).tobytes() + np.float32(0.0).tobytes()] +
                     [np.asarray(raw[k], np.float32) for k in keys])
    p = Params(nx=32, periodic=1, lado0=64.0, rmin=2.0, rmin_sub=2.0)
    out = run_iteration(path, p, tmp_path / "out", it=1, nlev=2, cubes=True, maps=True, engine=OracleEngine())
    head, levels = _read_voids_file(out["voids"])
    assert head["nlev"] == 2 and head["levmin"] == 0 and head["levmax"] == 1 and head["nmax"] == 32
    # level 0 is the oracle's level on the same particles in reader units
    parts = synth.to_reader_units({k: np.asarray(raw[k], np.float32) for k in keys})
    r0 = O.run_level(p, parts)
    l0, l1 = levels
    assert (l0["level"], l0["ncubes"], l0["nvoids"]) == (0, r0["vf"]["nvoid"], r0["cat"]["nvoidt"])
    # level 1: twice the grid, parents from level 0
    assert l1["level"] == 1 and l1["nparents"] == r0["vf"]["nvoid"]
    res1 = out["levels"][1]
    assert l1["ncubes"] == res1["nvoid"] and np.all(np.asarray(res1["cubes"]["father"]) > 0)
    _, reqp = O.next_level(p, r0["vf"]["nvoid"], r0["cat"]["marca"], r0["cat"]["uvoid"], r0["cat"]["req"])
    assert l1["nvoids"] > 0
    assert np.all(l1["rows"][:, 12] > 0)
    assert np.array_equal(l1["rows"][:, 13], reqp[l1["rows"][:, 12].astype(int) - 1])
    # the map holds both levels: 3 arrays of 32^3 then of 64^3 cells, 4 bytes each
    assert os.path.getsize(out["map"]) == 3 * 4 * (32 ** 3 + 64 ** 3)


class OracleModes(OracleEngine):
    def run_level_grid(self, p, nhy, u1, u2, u3, u4):
        return self._res(O.run_level_grid(p, nhy, u1, u2, u3, u4))

    def run_level_survey(self, p, parts, rands, smask):
        return self._res(O.run_level_survey(p, parts, rands, smask))

    def run_level_masclet(self, p, nhy, gas, parts, amr=None, want_marca=False):
        return self._res(O.run_level_masclet(p, nhy, gas, parts, amr))

    def run_sublevel_masclet(self, p, nhy, gas, marcap, reqp, parts, amr=None, want_marca=False):
        return self._res(O.run_sublevel_masclet(p, nhy, gas, marcap, reqp, parts, amr))

    def masclet_fields(self, p, nhy, gas, parts, amr=None):
        return O.masclet_fields(p, nhy, gas, parts, amr)


def test_grid_file_level(tmp_path):
    """A READ_BINARY_GRID file through the runner's grid mode (level -1)."""
    from avism_b200.run import run_single
    from test_grid_input import grid_case
    from avism_b200._abi import UV
    u1, vs = grid_case(32)
    path = tmp_path / "bin_file_grid00001"
    _fortran_records(path, [np.float32(0.0).tobytes(), (u1 - np.float32(1)).astype(np.float32)] +
                     [(v * np.float32(UV)).astype(np.float32) for v in vs])
    p = Params(nx=16, periodic=1, lado0=100.0, level=-1, levmin=-1, rmin=2.0)
    r = run_single(path, p, tmp_path / "out", grid_nhy=32, cubes=True, engine=OracleModes())
    head, levels = _read_voids_file(r["voids"])
    assert levels[0]["level"] == -1 and len(levels[0]["rows"]) == r["levels"][0]["cat"]["nvoidt"] > 0


def test_survey_files_level(tmp_path):
    """A particle file without velocities, mask.dat and rands.dat through the
    runner's survey mode."""
    from avism_b200.run import run_single
    c = synth.weighted_cone(box=150.0, ng=64, rmax=75.0, rsel=50.0, n_target=20000, seed=1005)
    rr = synth.cone_randoms(60000, c["pixel_mask"], box=150.0, rmax=75.0, rsel=50.0, seed=2005)
    sm = synth.cone_mask(64, c["pixel_mask"], box=150.0, rmax=75.0)
    pp = tmp_path / "bin_file_part00001"
    n = len(c["x"])
    _fortran_records(pp, [np.int64(n).tobytes() + np.float32(0.0).tobytes()] +
                     [c[k] for k in ("x", "y", "z", "m")])
    mp = tmp_path / "mask.dat"
    with open(mp, "wb") as f:
        f.write(np.int32(64).tobytes() + np.zeros(3, np.float32).tobytes() + sm.tobytes())
    rp = tmp_path / "rands.dat"
    _fortran_records(rp, [np.int32(len(rr["x"])).tobytes()] + [rr[k] for k in ("x", "y", "z", "w")])
    p = Params(nx=64, periodic=0, lado0=150.0, kneighbours=16, flag_vel_interp=0, flag_dens_interp=0, rmin=3.0)
    r = run_single(pp, p, tmp_path / "out", mask=mp, randoms=rp, novel=True, engine=OracleModes())
    head, levels = _read_voids_file(r["voids"])
    assert len(levels[0]["rows"]) == r["levels"][0]["cat"]["nvoidt"] > 0


def test_masclet_files_level(tmp_path):
    """A MASCLET snapshot's three files through the runner's MASCLET mode."""
    from avism_b200.run import run_single
    import masclet_case as mc
    snap = mc.snapshot()
    grid, gas, dm = mc.write_files(snap, str(tmp_path))
    p = Params(nx=snap["ng"], periodic=1, lado0=snap["box"], flag_dens=0, flag_div=0)
    r = run_single(grid, p, tmp_path / "out", masclet=(gas, dm), masclet_nhy=snap["ng"], cubes=True,
                   engine=OracleModes())
    head, levels = _read_voids_file(r["voids"])
    assert len(levels[0]["rows"]) == r["levels"][0]["cat"]["nvoidt"] > 0


def test_masclet_files_level1(tmp_path):
    """Level 1 of a MASCLET snapshot through the runner: the gas from the
    level-1 patches the reader takes from the grid and gas files."""
    from avism_b200.run import run_single
    import masclet_case as mc
    snap = mc.snapshot()
    grid, gas, dm = mc.write_files(snap, str(tmp_path))
    p = Params(nx=2 * snap["ng"], periodic=1, lado0=snap["box"], level=1, levmin=1, flag_dens=2, flag_div=2)
    r = run_single(grid, p, tmp_path / "out", masclet=(gas, dm), masclet_nhy=snap["ng"], cubes=True,
                   engine=OracleModes())
    o = O.run_level_masclet(p, snap["ng"], mc.gas(snap), None, mc.amr(snap))
    head, levels = _read_voids_file(r["voids"])
    assert len(levels[0]["rows"]) == r["levels"][0]["cat"]["nvoidt"] == o["cat"]["nvoidt"] > 0


def test_masclet_two_levels(tmp_path):
    """Levels 0 and 1 of a MASCLET snapshot through the runner: level 1 inside
    the level-0 voids, from the level-1 patches; the files hold both levels and
    the map."""
    from avism_b200.run import run_masclet_iteration
    import masclet_case as mc
    snap = mc.snapshot()
    grid, gas, dm = mc.write_files(snap, str(tmp_path))
    p = Params(nx=snap["ng"], periodic=1, lado0=snap["box"], level=0, levmin=0, flag_dens=2, flag_div=2)
    r = run_masclet_iteration(grid, gas, dm, snap["ng"], p, tmp_path / "out", nlev=2, cubes=True, maps=True,
                              engine=OracleModes())
    head, levels = _read_voids_file(r["voids"])
    assert len(levels) == 2
    for lv, res in zip(levels, r["levels"]):
        assert len(lv["rows"]) == res["cat"]["nvoidt"] > 0
    assert os.path.getsize(r["map"]) > 0

