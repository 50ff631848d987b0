"""Writes the golden fixtures of tests/test_golden.py and
tests/test_gpu_config2.py from the CPU oracle.

The reference (Fortran, no compiler in this image) cannot produce outputs
here, so these fixtures freeze the oracle's results on small seeded inputs:
a change in the oracle or in the CUDA path that alters any of them shows up
as a test failure.  Run from the repository root:

    python tests/golden/make_golden.py            # the small fixtures
    python tests/golden/make_golden.py config2    # the 256^3 digests (minutes)
    python tests/golden/make_golden.py masclet    # the MASCLET snapshot's levels 0 and 1
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from avism_b200 import synth  # noqa: E402
from avism_b200._abi import Params  # noqa: E402
from oracle import oracle as O  # noqa: E402


def level_case():
    parts = synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=64.0, nsph=3, rmin=5.0, rmax=9.0, seed=7))
    out = {}
    for per in (1, 0):
        p = Params(nx=32, periodic=per, lado0=64.0)
        r = O.run_level(p, parts)
        out[f"p{per}_nvoid"] = np.int32(r["vf"]["nvoid"])
        out[f"p{per}_meandens"] = np.float32(r["meandens"])
        for k, v in r["vf"]["cubes"].items():
            out[f"p{per}_cube_{k}"] = np.asarray(v)
        for k in ("indice", "uvoid", "ncellv", "volnew", "req", "gxc", "gyc", "gzc", "xc", "yc", "zc"):
            out[f"p{per}_cat_{k}"] = np.asarray(r["cat"][k])
        out[f"p{per}_nvoidt"] = np.int32(r["cat"]["nvoidt"])
        out[f"p{per}_u_mass"] = np.asarray(r["grid"]["u_mass"])
    return out


def knn_case():
    rng = np.random.default_rng(20261203)
    x, y, z = (rng.uniform(-25, 25, 3000).astype(np.float32) for _ in range(3))
    qx, qy, qz = (rng.uniform(-25, 25, 500).astype(np.float32) for _ in range(3))
    out = {"x": x, "y": y, "z": z, "qx": qx, "qy": qy, "qz": qz}
    for L in (50.0, 0.0):
        i, d = O.knn(x, y, z, qx, qy, qz, 8, L)
        tag = "per" if L > 0 else "open"
        out[f"{tag}_idx"] = np.asarray(i)
        out[f"{tag}_dist"] = np.asarray(d)
    return out


def indexx_case():
    rng = np.random.default_rng(5)
    a = rng.integers(0, 40, 2000).astype(np.float32)          # many equal keys
    return {"arr": a, "indx": np.asarray(O.indexx(a))}


def digest(a) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def config2_input():
    """The 256^3 scale-up workload: 2^24 particles Poisson-sampled from a
    lognormal field (GRF on 256^3, P(k) ~ k^-1.5, sigma_ln = 1), periodic
    L = 250 cMpc, linear-theory velocities at 350 km/s rms, seed 1002."""
    return synth.to_reader_units(synth.lognormal(n=2 ** 24, ng=256, box=250.0, index=-1.5, sigma_ln=1.0,
                                                 vrms=350.0, seed=1002))


CONFIG2_CAT = ("indice", "uvoid", "ncellv", "volnew", "req", "xc", "yc", "zc", "gxc", "gyc", "gzc", "eps", "ip",
               "umean", "mtot")


def config2_case():
    """Digests of the oracle's fields, cubes and catalogue at 256^3 for SPH/SPH
    and TSC/TSC (k = 32, README thresholds), and the catalogue columns."""
    parts = config2_input()
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")
    out = {"input": np.array(digest(np.concatenate([parts[k] for k in keys])))}
    for vel, dens in ((1, 1), (0, 0)):
        tag = f"v{vel}d{dens}"
        p = Params(nx=256, periodic=1, lado0=250.0, kneighbours=32, flag_vel_interp=vel, flag_dens_interp=dens,
                   nvoid_max=4_000_000)
        r = O.run_level(p, parts)
        for k in ("u_mass", "u2", "u3", "u4", "hpart", "part_dens"):
            out[f"{tag}_{k}"] = np.array(digest(r["grid"][k]))
        out[f"{tag}_u1co"] = np.array(digest(r["u1co"]))
        out[f"{tag}_diverco"] = np.array(digest(r["diverco"]))
        out[f"{tag}_meandens"] = np.float32(r["meandens"])
        out[f"{tag}_nvoid"] = np.int32(r["vf"]["nvoid"])
        out[f"{tag}_cubes"] = np.array(digest(np.concatenate([np.asarray(r["vf"]["cubes"][k]).view(np.int32)
                                                              for k in sorted(r["vf"]["cubes"])])))
        out[f"{tag}_marca"] = np.array(digest(r["cat"]["marca"]))
        for k in CONFIG2_CAT:
            out[f"{tag}_cat_{k}"] = np.asarray(r["cat"][k])
        out[f"{tag}_nvoidt"] = np.int32(r["cat"]["nvoidt"])
        print(tag, r["vf"]["nvoid"], r["cat"]["nvoidt"], flush=True)
    return out


MASCLET_CAT = ("indice", "uvoid", "ncellv", "volnew", "req", "gxc", "gyc", "gzc", "eps", "ip", "umean", "mtot")


def masclet_case():
    """The seeded MASCLET snapshot of tests/masclet_case.py (32^3 gas, DM
    particles on three levels, four level-1 patches): level 0 with FLAG_DENS =
    0 (DM + gas) and FLAG_DIV = -1 (linear theory), and level 1 inside the
    level-0 voids with FLAG_DENS = 0 and FLAG_DIV = 2 (the patches' gas
    divergence); field digests, cubes and catalogue columns."""
    sys.path.insert(0, os.path.dirname(HERE))
    import masclet_case as mc
    s = mc.snapshot()
    ng = s["ng"]
    out = {}
    p0 = Params(nx=ng, periodic=1, lado0=s["box"], level=0, levmin=0, flag_dens=0, flag_div=-1)
    r0 = O.run_level_masclet(p0, ng, mc.gas(s), mc.particles(s))
    mp, rq = O.next_level(p0, r0["vf"]["nvoid"], r0["cat"]["marca"], r0["cat"]["uvoid"], r0["cat"]["req"])
    p1 = Params(nx=2 * ng, periodic=1, lado0=s["box"], level=1, levmin=0, flag_dens=0, flag_div=2)
    r1 = O.run_sublevel_masclet(p1, ng, mc.gas(s), mp, rq, mc.particles(s), mc.amr(s))
    for tag, r in (("l0", r0), ("l1", r1)):
        out[f"{tag}_u1co"] = np.array(digest(r["u1co"]))
        out[f"{tag}_diverco"] = np.array(digest(r["diverco"]))
        out[f"{tag}_meandens"] = np.float32(r["meandens"])
        out[f"{tag}_nvoid"] = np.int32(r["vf"]["nvoid"])
        out[f"{tag}_cubes"] = np.array(digest(np.concatenate([np.asarray(r["vf"]["cubes"][k]).view(np.int32)
                                                              for k in sorted(r["vf"]["cubes"])])))
        for k in MASCLET_CAT:
            out[f"{tag}_cat_{k}"] = np.asarray(r["cat"][k])
        out[f"{tag}_nvoidt"] = np.int32(r["cat"]["nvoidt"])
        print(tag, r["vf"]["nvoid"], r["cat"]["nvoidt"], flush=True)
    return out


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "masclet":
        np.savez_compressed(os.path.join(HERE, "masclet32.npz"), **masclet_case())
        print("written")
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "config2":
        np.savez_compressed(os.path.join(HERE, "config2_256.npz"), **config2_case())
        print("written")
        sys.exit(0)
    np.savez_compressed(os.path.join(HERE, "level_mock32.npz"), **level_case())
    np.savez_compressed(os.path.join(HERE, "knn_3000.npz"), **knn_case())
    np.savez_compressed(os.path.join(HERE, "indexx_ties.npz"), **indexx_case())
    print("written")
