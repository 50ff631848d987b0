"""Standalone run of one iteration without the Fortran driver.

A READ_BINARY_PART_1 particle file in; the voids, cubes and map files of the
iteration out, for levels LEVMIN..LEVMAX (each level at twice the previous
grid, inside the previous level's voids), in the layout tools/read_voids.py
reads.  It is the reference's level loop (src/avism.f90:742-2181) for particle
input, with the particle arrays kept across levels::

    python -m avism_b200.run input_data/bin_file_part00001 --nx 64 --lado0 100 \\
        --levels 2 --out output_files --iter 1 --cubes --map

Masses and velocities are divided by UM and UV after reading, as
src/reader.f90:455-458 does.  The work runs on the GPU through the C-ABI.

The reference's other inputs, one level each:
  * --grid NHY: a READ_BINARY_GRID file (delta and velocities on NHY^3 cells,
    src/reader.f90:523-552) at the level with --nx = NHY * 2^level, level <= 0;
  * --mask FILE --randoms FILE: survey mode (FLAG_SURVEY = 1) with the mask and
    randoms files (src/avism.f90:403-418, 1425-1444); --novel reads the
    particle file as READ_BINARY_PART_2 (no velocities);
  * --masclet GAS DM --nhy NHYX: a MASCLET snapshot (the positional file is its
    grid file); with --levels 2 and --level 0, level 1 runs inside the level-0
    voids from the snapshot's level-1 patches.
"""
from __future__ import annotations

import argparse
import os

from ._abi import Params
from .avism import append_catalogue_level, read_particle_file, write_catalogue_headers


def run_iteration(particle_path, p: Params, out_dir, it: int = 1, nlev: int = 1, cubes: bool = False,
                  maps: bool = False, engine=None) -> dict:
    """Run levels p.levmin .. p.levmin + nlev - 1 and write their files; returns
    the paths and each level's result.  ``engine`` is an AvismGPU (default:
    device 0) or anything with its run_level / run_sublevel / next_level /
    particles_to_grid / fields methods."""
    from . import synth
    parts = read_particle_file(particle_path)
    p = Params(**{**p.__dict__, "zeta": float(parts.pop("zeta")), "level": p.levmin})
    parts = synth.to_reader_units(parts)
    if engine is None:
        from .avism import AvismGPU
        engine = AvismGPU(0)
        if p.learned == 1:
            from . import proposal
            engine.proposal_load(proposal.load_weights())
    os.makedirs(out_dir, exist_ok=True)
    vp = os.path.join(out_dir, f"voids{it:05d}")
    cp = os.path.join(out_dir, f"cubes{it:05d}") if cubes else None
    mp = os.path.join(out_dir, f"map{it:05d}") if maps else None
    write_catalogue_headers(vp, cp, nlev, p.levmin, p.levmin + nlev - 1, p.nx, p.nx, p.nx, p.lado0)
    if mp:
        open(mp, "wb").close()
    results = []
    req_parent, nvoidp, marcap, reqp = None, 0, None, None
    for lev in range(nlev):
        q = Params(**{**p.__dict__, "nx": p.nx * 2 ** lev, "level": p.levmin + lev})
        keep_marca = maps or lev + 1 < nlev
        if lev == 0:
            res = engine.run_level(q, parts, want_marca=keep_marca)
        else:
            res = engine.run_sublevel(q, parts, marcap, reqp, want_marca=keep_marca)
        u1 = dv = None
        if maps:
            grid = engine.particles_to_grid(q, parts)
            u1, dv, _ = engine.fields(q, grid["u_mass"], grid["u2"], grid["u3"], grid["u4"])
        append_catalogue_level(vp, q, res, nvoidp=nvoidp, req_parent=req_parent, cubes_path=cp, map_path=mp,
                               u1co_ext=u1, diverco_ext=dv)
        results.append(res)
        if lev + 1 < nlev:
            cat = res["cat"]
            marcap, reqp = engine.next_level(q, res["nvoid"], cat["marca"], cat["uvoid"], cat["req"])
            req_parent, nvoidp = reqp, res["nvoid"]          # REQP and NVOIDP = NVOID (avism.f90:2139-2146)
    return dict(voids=vp, cubes=cp, map=mp, levels=results)


def run_masclet_iteration(grid_path, gas_path, dm_path, nhy, p: Params, out_dir, it: int = 1, nlev: int = 1,
                          cubes: bool = False, maps: bool = False, engine=None) -> dict:
    """A MASCLET snapshot's levels p.levmin .. p.levmin + nlev - 1 (at most level
    1; p.nx is the first level's grid, nhy * 2^levmin): the first with
    run_level_masclet, each next one inside the previous level's voids with
    run_sublevel_masclet, level 1 from the snapshot's level-1 patches, as the
    reference's level loop runs MASCLET input (src/avism.f90:742-2181)."""
    from .avism import read_masclet_files
    r = read_masclet_files(grid_path, gas_path, dm_path, nhy)
    p = Params(**{**p.__dict__, "zeta": float(r["zeta"]), "level": p.levmin})
    gas = tuple(r["gas"][k] for k in ("u1g", "u2g", "u3g", "u4g"))
    parts = r["parts"] if p.flag_dens <= 1 or p.flag_div in (0, 1) else None
    if engine is None:
        from .avism import AvismGPU
        engine = AvismGPU(0)
    os.makedirs(out_dir, exist_ok=True)
    vp = os.path.join(out_dir, f"voids{it:05d}")
    cp = os.path.join(out_dir, f"cubes{it:05d}") if cubes else None
    mp = os.path.join(out_dir, f"map{it:05d}") if maps else None
    write_catalogue_headers(vp, cp, nlev, p.levmin, p.levmin + nlev - 1, p.nx, p.nx, p.nx, p.lado0)
    if mp:
        open(mp, "wb").close()
    results = []
    req_parent, nvoidp, marcap, reqp = None, 0, None, None
    for lev in range(nlev):
        q = Params(**{**p.__dict__, "nx": p.nx * 2 ** lev, "level": p.levmin + lev})
        amr = r["amr"] if q.level == 1 else None
        keep_marca = maps or lev + 1 < nlev
        if lev == 0:
            res = engine.run_level_masclet(q, nhy, gas, parts, amr, want_marca=keep_marca)
        else:
            res = engine.run_sublevel_masclet(q, nhy, gas, marcap, reqp, parts, amr, want_marca=keep_marca)
        u1 = dv = None
        if maps:
            u1, dv, _ = engine.masclet_fields(q, nhy, gas, parts, amr)
        append_catalogue_level(vp, q, res, nvoidp=nvoidp, req_parent=req_parent, cubes_path=cp, map_path=mp,
                               u1co_ext=u1, diverco_ext=dv)
        results.append(res)
        if lev + 1 < nlev:
            cat = res["cat"]
            marcap, reqp = engine.next_level(q, res["nvoid"], cat["marca"], cat["uvoid"], cat["req"])
            req_parent, nvoidp = reqp, res["nvoid"]
    return dict(voids=vp, cubes=cp, map=mp, levels=results)


def run_single(path, p: Params, out_dir, it: int = 1, grid_nhy: int = 0, mask=None, randoms=None,
               novel: bool = False, ncox: int = 0, cubes: bool = False, engine=None, masclet=None,
               masclet_nhy: int = 0) -> dict:
    """One level from a grid file (grid_nhy > 0), a MASCLET snapshot (path the
    grid file, masclet = (gas file, DM file), masclet_nhy the base grid; level
    <= 1, level 1 from the snapshot's level-1 patches) or a survey (mask and randoms files), written as run_iteration writes
    its levels."""
    import numpy as np
    from . import synth
    from ._abi import UM, UV
    from .avism import (read_grid_file, read_mask_file, read_masclet_files, read_particle_file_novel,
                        read_randoms_file)
    if engine is None:
        from .avism import AvismGPU
        engine = AvismGPU(0)
    if grid_nhy:
        g = read_grid_file(path, grid_nhy)
        p = Params(**{**p.__dict__, "zeta": float(g["zeta"])})
        # delta -> rho / rho_B, km/s -> c (src/reader.f90:546-550)
        u1 = (g["u1"] + np.float32(1.0)).astype(np.float32)
        vs = [(g[k] / np.float32(UV)).astype(np.float32) for k in ("u2", "u3", "u4")]
        res = engine.run_level_grid(p, grid_nhy, u1, *vs)
    elif masclet:
        r = read_masclet_files(path, masclet[0], masclet[1], masclet_nhy)
        p = Params(**{**p.__dict__, "zeta": float(r["zeta"])})
        gas = tuple(r["gas"][k] for k in ("u1g", "u2g", "u3g", "u4g"))
        res = engine.run_level_masclet(p, masclet_nhy, gas, r["parts"], r["amr"] if p.level == 1 else None)
    else:
        parts = read_particle_file_novel(path) if novel else read_particle_file(path)
        p = Params(**{**p.__dict__, "zeta": float(parts.pop("zeta")), "no_velocities": int(novel)})
        parts = synth.to_reader_units(parts) if not novel else {**parts, "m": (parts["m"] / UM).astype(np.float32)}
        sm, _ = read_mask_file(mask, ncox or p.nx, p.nx)
        rr = read_randoms_file(randoms)
        rr["w"] = (rr["w"] / UM).astype(np.float32)            # MASSRAND / UM (src/avism.f90:1440)
        res = engine.run_level_survey(p, parts, rr, sm)
    os.makedirs(out_dir, exist_ok=True)
    vp = os.path.join(out_dir, f"voids{it:05d}")
    cp = os.path.join(out_dir, f"cubes{it:05d}") if cubes else None
    write_catalogue_headers(vp, cp, 1, p.level, p.level, p.nx, p.nx, p.nx, p.lado0)
    append_catalogue_level(vp, p, res, cubes_path=cp)
    return dict(voids=vp, cubes=cp, levels=[res])


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("particles")
    ap.add_argument("--nx", type=int, required=True)
    ap.add_argument("--lado0", type=float, required=True)
    ap.add_argument("--periodic", type=int, default=1)
    ap.add_argument("--kneighbours", type=int, default=32)
    ap.add_argument("--levels", type=int, default=1)
    ap.add_argument("--learned", type=int, default=0, choices=[0, 1, 2])
    ap.add_argument("--nvoid-max", type=int, default=4_000_000)
    ap.add_argument("--out", default="output_files")
    ap.add_argument("--iter", type=int, default=1)
    ap.add_argument("--cubes", action="store_true")
    ap.add_argument("--map", action="store_true")
    ap.add_argument("--grid", type=int, default=0, metavar="NHY", help="the input is a grid file of NHY^3 cells")
    ap.add_argument("--level", type=int, default=0, help="the level of a grid input (<= 0)")
    ap.add_argument("--mask", help="survey mask file (survey mode)")
    ap.add_argument("--randoms", help="survey randoms file (survey mode)")
    ap.add_argument("--ncox", type=int, default=0, help="the survey mask's coarse grid (default --nx)")
    ap.add_argument("--novel", action="store_true", help="particle file without velocities (READ_BINARY_PART_2)")
    ap.add_argument("--masclet", nargs=2, metavar=("GAS", "DM"),
                    help="the input (positional) is a MASCLET grid file with these gas and DM files")
    ap.add_argument("--nhy", type=int, default=0, help="the MASCLET base grid (NHYX)")
    ap.add_argument("--flag-dens", type=int, default=0, choices=[0, 1, 2], help="MASCLET FLAG_DENS")
    ap.add_argument("--flag-div", type=int, default=0, choices=[-1, 0, 1, 2], help="MASCLET FLAG_DIV")
    a = ap.parse_args(argv)
    p = Params(nx=a.nx, lado0=a.lado0, periodic=a.periodic, kneighbours=a.kneighbours, learned=a.learned,
               nvoid_max=a.nvoid_max, level=a.level, levmin=a.level, flag_dens=a.flag_dens, flag_div=a.flag_div)
    if a.masclet and a.levels > 1:
        r = run_masclet_iteration(a.particles, a.masclet[0], a.masclet[1], a.nhy or a.nx, p, a.out, it=a.iter,
                                  nlev=a.levels, cubes=a.cubes, maps=a.map)
    elif a.grid or a.mask or a.masclet:
        r = run_single(a.particles, p, a.out, it=a.iter, grid_nhy=a.grid, mask=a.mask, randoms=a.randoms,
                       novel=a.novel, ncox=a.ncox, cubes=a.cubes, masclet=a.masclet, masclet_nhy=a.nhy or a.nx)
    else:
        r = run_iteration(a.particles, p, a.out, it=a.iter, nlev=a.levels, cubes=a.cubes, maps=a.map)
    for lev in r["levels"]:
        print(f"level: {lev['nvoid']} cubes, {lev['cat']['nvoidt']} voids")
    print(f"wrote {r['voids']}" + (f", {r['cubes']}" if r["cubes"] else "") +
          (f", {r['map']}" if r.get("map") else ""))


if __name__ == "__main__":
    main()
