"""GPU parity at the 256^3 scale-up configuration (2^24 lognormal particles,
P(k) ~ k^-1.5, periodic L = 250 cMpc, k = 32), SPH/SPH and TSC/TSC, against
the oracle's results frozen in tests/golden/config2_256.npz (written by
tests/golden/make_golden.py config2): SHA-256 digests of every field and of the
cube set, and the catalogue columns themselves."""
import hashlib
import os

import numpy as np
import pytest

from avism_b200._abi import Params

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config2_256.npz")
EXACT = ("indice", "uvoid", "ncellv", "volnew", "req", "xc", "yc", "zc", "gxc", "gyc", "gzc", "eps", "ip", "umean",
         "mtot")


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def case():
    import sys
    sys.path.insert(0, os.path.dirname(GOLD))
    import make_golden
    gold = dict(np.load(GOLD))
    parts = make_golden.config2_input()
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")
    assert digest(np.concatenate([parts[k] for k in keys])) == str(gold["input"]), "input generator changed"
    return gold, parts


@pytest.mark.parametrize("vel,dens", [(1, 1), (0, 0)])
def test_config2_level_matches_oracle(gpu, case, vel, dens):
    gold, parts = case
    tag = f"v{vel}d{dens}"
    p = Params(nx=256, periodic=1, lado0=250.0, kneighbours=32, flag_vel_interp=vel, flag_dens_interp=dens,
               nvoid_max=4_000_000)
    g = gpu.particles_to_grid(p, parts)
    for k in ("u_mass", "u2", "u3", "u4", "hpart", "part_dens"):
        assert digest(g[k]) == str(gold[f"{tag}_{k}"]), k
    u1, dv, md = gpu.fields(p, g["u_mass"], g["u2"], g["u3"], g["u4"])
    assert digest(u1) == str(gold[f"{tag}_u1co"]) and digest(dv) == str(gold[f"{tag}_diverco"])
    assert md == gold[f"{tag}_meandens"]
    r = gpu.run_level(p, parts, capacity=4_000_000, want_marca=True)
    assert r["nvoid"] == int(gold[f"{tag}_nvoid"])
    cubes = np.concatenate([np.asarray(r["cubes"][k]).view(np.int32) for k in sorted(r["cubes"])])
    assert digest(cubes) == str(gold[f"{tag}_cubes"])
    assert digest(r["cat"]["marca"]) == str(gold[f"{tag}_marca"])
    assert r["cat"]["nvoidt"] == int(gold[f"{tag}_nvoidt"]) > 0
    for k in EXACT:
        assert np.array_equal(np.asarray(r["cat"][k]), gold[f"{tag}_cat_{k}"]), k
