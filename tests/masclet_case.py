"""Seeded synthetic MASCLET snapshots for the tests: the level-0 gas grids (a
lognormal density contrast and linear-theory velocities), dark-matter particles
on level 0 (mass MAP) and on two refinement levels (their own masses), and a
writer of the three files READ_MASCLET reads (src/reader.f90:86-405): the grid
file (text) and the gas and dark-matter files (sequential unformatted, 4-byte
record markers).  The patches' grids are written as records of the right size
with arbitrary values; the library's reader skips them."""
import numpy as np

from avism_b200 import synth
from avism_b200._abi import UV


def snapshot(ng=32, box=64.0, seed=11):
    """(gas delta and velocities at ng^3 column-major, DM particles by level,
    patch sizes by level, MAP)."""
    rng = np.random.default_rng(seed)
    g, vel = synth._grf(ng, box, -1.5, 1.0, rng)
    rho = np.exp(g)
    rho /= rho.mean()
    cm = lambda a: np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()
    delta = (cm(rho) - 1.0).astype(np.float32)
    vs = [(cm(v * 300.0 / np.std(v)).astype(np.float32) / np.float32(UV)).astype(np.float32) for v in vel]
    base = synth.to_reader_units(synth.mock_spheres(n=2 ** 14, box=box, nsph=3, rmin=5.0, rmax=9.0, seed=seed))
    n0 = 2 ** 13
    mp = np.float32(base["m"][0])
    lev0 = {k: base[k][:n0].copy() for k in ("x", "y", "z", "vx", "vy", "vz")}
    lev = []
    cut = [n0, n0 + 5000, 2 ** 14]
    for i in range(2):
        sl = slice(cut[i], cut[i + 1])
        d = {k: base[k][sl].copy() for k in ("x", "y", "z", "vx", "vy", "vz")}
        d["m"] = (base["m"][sl] * np.float32(0.125 ** (i + 1))).astype(np.float32)
        lev.append(d)
    patches = [[(8, 6, 10), (4, 4, 4)], [(6, 6, 6)]]
    return dict(ng=ng, box=box, delta=delta, vel=vs, lev0=lev0, lev=lev, map=mp, patches=patches)


def _rec(f, a):
    b = np.ascontiguousarray(a).tobytes()
    hdr = np.int32(len(b)).tobytes()
    f.write(hdr + b + hdr)


def write_files(s, folder, zeta=0.0):
    """The grid, gas and DM files of snapshot s; returns their paths."""
    import os
    grid, gas, dm = (os.path.join(folder, n) for n in ("grids00001", "clus00001", "cldm00001"))
    nl = len(s["lev"])
    with open(grid, "w") as f:
        f.write(f"1 0.5 {nl} {float(s['map']):.9g}\n{zeta:.6f}\n0 {len(s['lev0']['x'])} 0\n")
        for ir in range(1, nl + 1):
            pl = s["patches"][ir - 1]
            f.write(f"{ir} {len(pl)} {len(s['lev'][ir - 1]['x'])} 0\n")
            f.write("  patch data\n")
            for j, (a, b, c) in enumerate(pl):
                f.write(f"{a} {b} {c}\n{3 + j} 5 7\n{0.25:.6f}, {-1.5:.6f}, {2.0:.6f}\n{j}\n")
    ng3 = s["ng"] ** 3
    with open(gas, "wb") as f:
        _rec(f, np.array([1, 0], np.int32))
        for a in [s["delta"]] + s["vel"]:
            _rec(f, a.astype(np.float32))
        for _ in range(6):
            _rec(f, np.zeros(ng3, np.float32))
        for pl in s["patches"]:
            for (a, b, c) in pl:
                for _ in range(11):
                    _rec(f, np.full(a * b * c, 7.0, np.float32))
    with open(dm, "wb") as f:
        _rec(f, np.array([1, 0], np.int32))
        _rec(f, np.zeros(ng3, np.float32))
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            _rec(f, s["lev0"][k].astype(np.float32))
        _rec(f, np.arange(len(s["lev0"]["x"]), dtype=np.int32))
        for ir, pl in enumerate(s["patches"]):
            for (a, b, c) in pl:
                _rec(f, np.full(a * b * c, 3.0, np.float32))
            for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
                _rec(f, s["lev"][ir][k].astype(np.float32))
            _rec(f, np.arange(len(s["lev"][ir]["x"]), dtype=np.int32))
    return grid, gas, dm


def particles(s):
    """Every level's particles as READ_MASCLET concatenates them."""
    out = {}
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        out[k] = np.concatenate([s["lev0"][k]] + [d[k] for d in s["lev"]]).astype(np.float32)
    out["m"] = np.concatenate([np.full(len(s["lev0"]["x"]), s["map"], np.float32)] +
                              [d["m"] for d in s["lev"]]).astype(np.float32)
    return out


def gas(s):
    """(U1G = delta + 1, U2G, U3G, U4G) as the reader leaves them."""
    return ((s["delta"] + np.float32(1.0)).astype(np.float32), *s["vel"])
