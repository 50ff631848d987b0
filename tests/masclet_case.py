"""Seeded synthetic MASCLET snapshots for the tests: the level-0 gas grids (a
lognormal density contrast and linear-theory velocities), dark-matter particles
on level 0 (mass MAP) and on two refinement levels (their own masses), and a
writer of the three files READ_MASCLET reads (src/reader.f90:86-405): the grid
file (text) and the gas and dark-matter files (sequential unformatted, 4-byte
record markers).  Level 1 carries four patches with their own gas cells (two of
them overlapping, one of odd sizes, one near the base grid's edge), placed the
way VMESH (src/amr2uniform.f90:170-172) maps them onto the level-1 grid; level
2's patch grids are records of the right size with arbitrary values."""
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
    amr = _level1_patches(ng, box, delta, vs, rng)
    patches = [[tuple(int(amr[k][i]) for k in ("nx", "ny", "nz")) for i in range(len(amr["nx"]))], [(6, 6, 6)]]
    return dict(ng=ng, box=box, delta=delta, vel=vs, lev0=lev0, lev=lev, map=mp, patches=patches, amr=amr)


# level-1 patches: sizes and first base cells (1-based)
_L1 = [((8, 6, 10), (5, 9, 4)), ((4, 4, 4), (7, 10, 6)), ((7, 5, 9), (20, 22, 25)), ((3, 4, 5), (2, 2, 27))]


def _level1_patches(ng, box, delta, vel, rng):
    """Patches of _L1 at level 1 (cells of half the base size): the first cell
    of a patch whose first base cell is l sits at level-1 index 2(l - 1) + 1;
    the corner PATCHRX is chosen so that VMESH's
    INT(((RX - DXR/2) - RX1)/DXR + 0.5) gives 2(l - 1).  The cells take the
    parent base cell's delta and velocities with noise."""
    from oracle import oracle as O
    from avism_b200._abi import Params
    f32 = np.float32
    g, rad = O.grid_setup(Params(nx=2 * ng, periodic=1, lado0=box, level=1, levmin=1))
    dxr, rx1 = f32(g.dx), f32(rad[1 - g.rad_lo])
    out = {k: [] for k in ("nx", "ny", "nz", "ix", "iy", "iz", "rx", "ry", "rz")}
    cells = {k: [] for k in ("d11", "u12g", "u13g", "u14g")}
    base = lambda a: a.reshape(ng, ng, ng)                  # [k, j, i] of the column-major grid
    for (n, l) in _L1:
        for a, key in enumerate(("nx", "ny", "nz")):
            out[key].append(n[a])
            out[("ix", "iy", "iz")[a]].append(l[a])
            want = 2 * (l[a] - 1)
            r = f32(rx1 + f32(f32(want) * dxr))
            got = int(f32(f32(f32(f32(r - f32(f32(0.5) * dxr)) - rx1) / dxr) + f32(0.5)))
            assert got == want, (r, got, want)
            out[("rx", "ry", "rz")[a]].append(r)
        # parent base cell of patch cell (i, j, k): (i + 1)//2 + l - 1 (1-based)
        kk, jj, ii = np.meshgrid(*[(np.arange(1, n[a] + 1) + 1) // 2 + l[a] - 2 for a in (2, 1, 0)], indexing="ij")
        for key, src, sc in (("d11", delta, 0.2), ("u12g", vel[0], 0.1), ("u13g", vel[1], 0.1),
                             ("u14g", vel[2], 0.1)):
            v = base(src)[kk, jj, ii]
            v = (v + sc * np.std(src) * rng.standard_normal(v.shape)).astype(f32)
            cells[key].append(np.ascontiguousarray(v).ravel())
    amr = {k: np.asarray(v, np.int32) for k, v in out.items() if k in ("nx", "ny", "nz", "ix", "iy", "iz")}
    amr.update({k: np.asarray(out[k], np.float32) for k in ("rx", "ry", "rz")})
    sizes = [a * b * c for (a, b, c), _ in _L1]
    amr["offset"] = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    amr["d11"] = np.maximum(np.concatenate(cells["d11"]), f32(-0.95)).astype(f32)
    amr["u11g"] = (amr["d11"] + f32(1.0)).astype(f32)
    for k in ("u12g", "u13g", "u14g"):
        amr[k] = np.concatenate(cells[k]).astype(f32)
    return amr


def amr(s):
    """The level-1 patches as the `amr` argument (U11G = delta + 1)."""
    return {k: v for k, v in s["amr"].items() if k != "d11"}


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
                if ir == 1:
                    am = s["amr"]
                    geo = " ".join(str(int(am[k][j])) for k in ("ix", "iy", "iz"))
                    cor = ", ".join(f"{float(am[k][j]):.9g}" for k in ("rx", "ry", "rz"))
                    f.write(f"{a} {b} {c}\n{geo}\n{cor}\n0\n")
                else:
                    f.write(f"{a} {b} {c}\n{3 + j} 5 7\n{0.25:.6f}, {-1.5:.6f}, {2.0:.6f}\n{j}\n")
    ng3 = s["ng"] ** 3
    with open(gas, "wb") as f:
        _rec(f, np.array([1, 0], np.int32))
        for a in [s["delta"]] + s["vel"]:
            _rec(f, a.astype(np.float32))
        for _ in range(6):
            _rec(f, np.zeros(ng3, np.float32))
        am = s["amr"]
        for ir, pl in enumerate(s["patches"]):
            for j, (a, b, c) in enumerate(pl):
                if ir == 0:
                    sl = slice(int(am["offset"][j]), int(am["offset"][j + 1]))
                    for k in ("d11", "u12g", "u13g", "u14g"):
                        _rec(f, am[k][sl])
                    for _ in range(7):
                        _rec(f, np.full(a * b * c, 7.0, np.float32))
                else:
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
