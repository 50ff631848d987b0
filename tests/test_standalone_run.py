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
