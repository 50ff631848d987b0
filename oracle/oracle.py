"""ctypes wrapper of the C oracle (oracle/liboracle.so) -- test infrastructure.

Parity unpinned by the reference: it cannot be built here (Fortran) and ships
no golden vectors; the oracle is pinned by known-answer cases instead.

Every function restates a reference routine; see the C sources for the
file:line each follows.  Arrays are numpy, grids Fortran column-major and
flattened (x fastest), index outputs keep the reference's values.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from avism_b200._abi import (AVISM_OK, AvismGrid, AvismParams, Cubes, Params, Voids,
                             STATUS_NAMES, ptr)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (make rebuilds it when a
    source or header is newer than the library)."""
    subprocess.run(["make", "-C", _HERE, "-B" if force else "liboracle.so"], check=True, capture_output=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
    return _lib


class OracleError(RuntimeError):
    pass


def _chk(st):
    if st != AVISM_OK:
        raise OracleError(f"oracle status {st} ({STATUS_NAMES.get(st, '?')})")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def grid_setup(p: Params):
    g = AvismGrid()
    pc = p.to_c()
    _chk(lib().orc_grid_setup(C.byref(pc), C.byref(g), None))
    rad = np.zeros(g.rad_hi - g.rad_lo + 1, np.float32)
    _chk(lib().orc_grid_setup(C.byref(pc), C.byref(g), ptr(rad, C.c_float)))
    return g, rad


def knn(x, y, z, qx, qy, qz, k, box_l=0.0):
    x, y, z, qx, qy, qz = map(_f32, (x, y, z, qx, qy, qz))
    nq = len(qx)
    idx = np.zeros(nq * k, np.int64)
    dist = np.zeros(nq * k, np.float32)
    f = lib().orc_knn
    f.argtypes = [C.c_int64] + [C.POINTER(C.c_float)] * 3 + [C.c_float, C.c_int64] + \
        [C.POINTER(C.c_float)] * 3 + [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_float)]
    _chk(f(len(x), ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float), box_l, nq,
           ptr(qx, C.c_float), ptr(qy, C.c_float), ptr(qz, C.c_float), k,
           ptr(idx, C.c_int64), ptr(dist, C.c_float)))
    return idx.reshape(nq, k), dist.reshape(nq, k)


def particles_to_grid(p: Params, x, y, z, vx, vy, vz, m, smask=None):
    # without velocities (no_velocities = 1) zeros stand in for them
    vx, vy, vz = (np.zeros(len(x), np.float32) if v is None else v for v in (vx, vy, vz))
    x, y, z, vx, vy, vz, m = map(_f32, (x, y, z, vx, vy, vz, m))
    n = len(x)
    nc = p.nx ** 3
    out = [np.zeros(nc, np.float32) for _ in range(4)]
    h = np.zeros(n, np.float32)
    pd = np.zeros(n, np.float32)
    f = lib().orc_particles_to_grid
    f.argtypes = [C.c_void_p, C.c_int64] + [C.POINTER(C.c_float)] * 7 + \
        [C.c_void_p] + [C.POINTER(C.c_float)] * 6
    pc = p.to_c()
    sm = None if smask is None else np.ascontiguousarray(smask, np.int8)
    _chk(f(C.byref(pc), n, *(ptr(a, C.c_float) for a in (x, y, z, vx, vy, vz, m)),
           None if sm is None else sm.ctypes.data, *(ptr(a, C.c_float) for a in out),
           ptr(h, C.c_float), ptr(pd, C.c_float)))
    return dict(u_mass=out[0], u2=out[1], u3=out[2], u4=out[3], hpart=h, part_dens=pd)


def path_counts():
    """(ball-fallback cells, FILL_H_ZEROS orphans, DDENS NORM = 0 particles) of
    the last particles_to_grid call."""
    out = np.zeros(3, np.int64)
    lib().orc_path_counts(out.ctypes.data_as(C.POINTER(C.c_int64)))
    return dict(ball_cells=int(out[0]), orphans=int(out[1]), norm0=int(out[2]))


def fields(p: Params, u_mass, u2, u3, u4):
    g, _ = grid_setup(p)
    u2, u3, u4 = (np.zeros(p.nx ** 3, np.float32) if v is None else v for v in (u2, u3, u4))
    ne3 = g.ne ** 3
    u1 = np.zeros(ne3, np.float32)
    dv = np.zeros(ne3, np.float32)
    md = C.c_float()
    f = lib().orc_fields
    f.argtypes = [C.c_void_p] + [C.POINTER(C.c_float)] * 6 + [C.POINTER(C.c_float)]
    pc = p.to_c()
    _chk(f(C.byref(pc), *(ptr(_f32(a), C.c_float) for a in (u_mass, u2, u3, u4)),
           ptr(u1, C.c_float), ptr(dv, C.c_float), C.byref(md)))
    return u1, dv, md.value


def survey_fields(p: Params, parts: dict, rands: dict, smask):
    """Survey mode (src/avism.f90:1420-1596): tracers and randoms to the grid,
    the D/(alpha R) contrast and the divergence; (U1CO ext, DIVERCO ext,
    MEANDENS, the randoms' grid)."""
    g, _ = grid_setup(p)
    n = len(parts["x"])
    zero = np.zeros(n, np.float32)
    a = [_f32(parts[k]) if parts.get(k) is not None else zero for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
    r = [_f32(rands[k]) for k in ("x", "y", "z", "w")]
    sm = np.ascontiguousarray(smask, np.int8)
    ne3 = g.ne ** 3
    u1 = np.zeros(ne3, np.float32)
    dv = np.zeros(ne3, np.float32)
    ur = np.zeros(p.nx ** 3, np.float32)
    md = C.c_float()
    f = lib().orc_survey_fields
    f.argtypes = [C.c_void_p, C.c_int64] + [C.POINTER(C.c_float)] * 7 + [C.c_int64] + \
        [C.POINTER(C.c_float)] * 4 + [C.c_void_p] + [C.POINTER(C.c_float)] * 3 + [C.POINTER(C.c_float)]
    pc = p.to_c()
    _chk(f(C.byref(pc), n, *(ptr(v, C.c_float) for v in a), len(r[0]), *(ptr(v, C.c_float) for v in r),
           sm.ctypes.data, ptr(u1, C.c_float), ptr(dv, C.c_float), C.byref(md), ptr(ur, C.c_float)))
    return u1, dv, md.value, ur


def grid_fields(p: Params, nhy, u1g, u2g, u3g, u4g):
    """Grid input (src/avism.f90:1316-1362): (U1CO ext, DIVERCO ext, MEANDENS)."""
    g, _ = grid_setup(p)
    u1 = np.zeros(g.ne ** 3, np.float32)
    dv = np.zeros(g.ne ** 3, np.float32)
    md = C.c_float()
    f = lib().orc_grid_fields
    f.argtypes = [C.c_void_p, C.c_int32] + [C.POINTER(C.c_float)] * 6 + [C.POINTER(C.c_float)]
    pc = p.to_c()
    _chk(f(C.byref(pc), int(nhy), *(ptr(_f32(a), C.c_float) for a in (u1g, u2g, u3g, u4g)),
           ptr(u1, C.c_float), ptr(dv, C.c_float), C.byref(md)))
    return u1, dv, md.value


def run_level_grid(p: Params, nhy, u1g, u2g, u3g, u4g):
    """grids -> catalogue on the CPU (grid input)."""
    u1, dv, md = grid_fields(p, nhy, u1g, u2g, u3g, u4g)
    vf = voidfind(p, u1, dv)
    cat = merge_post(p, vf["nvoid"], vf["cubes"], u1, md)
    return dict(u1co=u1, diverco=dv, meandens=md, vf=vf, cat=cat)


def masclet_fields(p: Params, nhy, gas, parts=None, amr=None):
    """MASCLET input at levels <= 0 (src/avism.f90:980-1156, 1366-1405,
    1633-1650): (U1CO ext, DIVERCO ext, MEANDENS) from the gas grids
    (u1g = 1 + delta, u2g, u3g, u4g at nhy^3) and the DM particles."""
    g, _ = grid_setup(p)
    u1 = np.zeros(g.ne ** 3, np.float32)
    dv = np.zeros(g.ne ** 3, np.float32)
    md = C.c_float()
    f = lib().orc_masclet_fields
    f.argtypes = [C.c_void_p, C.c_int32] + [C.POINTER(C.c_float)] * 4 + [C.c_void_p, C.c_int64] + \
        [C.POINTER(C.c_float)] * 7 + [C.POINTER(C.c_float)] * 3
    from avism_b200._abi import patches_c
    pa, keep_amr = patches_c(amr) if amr is not None else (None, None)
    keep = [None if a is None else _f32(a) for a in gas]
    gp = [ptr(a, C.c_float) if a is not None else None for a in keep]
    if parts is None:
        n, pp = 0, [None] * 7
    else:
        pk = [_f32(parts[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        n, pp = len(pk[0]), [ptr(a, C.c_float) for a in pk]
    pc = p.to_c()
    _chk(f(C.byref(pc), int(nhy), *gp, C.byref(pa) if pa is not None else None, n, *pp, ptr(u1, C.c_float),
           ptr(dv, C.c_float), C.byref(md)))
    return u1, dv, md.value


def run_level_masclet(p: Params, nhy, gas, parts=None, amr=None):
    """MASCLET snapshot level -> catalogue on the CPU."""
    u1, dv, md = masclet_fields(p, nhy, gas, parts, amr)
    vf = voidfind(p, u1, dv)
    cat = merge_post(p, vf["nvoid"], vf["cubes"], u1, md)
    return dict(u1co=u1, diverco=dv, meandens=md, vf=vf, cat=cat)


def run_sublevel_masclet(p: Params, nhy, gas, marcap_ext, reqp, parts=None, amr=None):
    """A MASCLET level inside the parent voids on the CPU."""
    u1, dv, md = masclet_fields(p, nhy, gas, parts, amr)
    vf = voidfind(p, u1, dv, marcap_ext=marcap_ext, reqp=reqp)
    cat = merge_post(p, vf["nvoid"], vf["cubes"], u1, md)
    return dict(u1co=u1, diverco=dv, meandens=md, vf=vf, cat=cat)


def smask_ext(p: Params, smask):
    """The survey mask on the ext grid: the inner cells' values, 0 on the ghost
    shell (SMASK = 0 before the inner cells are set, src/avism.f90:867-869)."""
    g, _ = grid_setup(p)
    ne, nx = g.ne, g.nx
    out = np.zeros((ne, ne, ne), np.int8)
    o = 1 - g.low1
    out[o:o + nx, o:o + nx, o:o + nx] = np.asarray(smask, np.int8).reshape(nx, nx, nx)
    return out.ravel()


def run_level_survey(p: Params, parts: dict, rands: dict, smask):
    """particles + randoms -> catalogue in survey mode on the CPU."""
    u1, dv, md, ur = survey_fields(p, parts, rands, smask)
    se = smask_ext(p, smask)
    vf = voidfind(p, u1, dv, smask_ext=se)
    cat = merge_post(p, vf["nvoid"], vf["cubes"], u1, md)
    return dict(u1co=u1, diverco=dv, meandens=md, u1rand=ur, vf=vf, cat=cat, smask_ext=se)


def diver_uniform(nx, dx, v2, v3, v4, periodic):
    out = np.zeros(nx ** 3, np.float32)
    f = lib().orc_diver_uniform
    f.argtypes = [C.c_int, C.c_float] + [C.POINTER(C.c_float)] * 3 + [C.c_int, C.POINTER(C.c_float)]
    _chk(f(nx, dx, *(ptr(_f32(a), C.c_float) for a in (v2, v3, v4)), periodic,
           ptr(out, C.c_float)))
    return out


def voidfind(p: Params, u1co_ext, diverco_ext, smask_ext=None, marcap_ext=None, reqp=None):
    g, _ = grid_setup(p)
    ne3 = g.ne ** 3
    u1 = _f32(u1co_ext)
    dv = _f32(diverco_ext)
    flags = np.zeros(ne3, np.uint8)
    cap = int(min(p.nvoid_max, max(ne3 // 8, 1024)))
    cubes = Cubes(cap)
    nvoid = C.c_int32()
    nc = C.c_int32()
    order = np.zeros(ne3, np.int32)
    f = lib().orc_voidfind
    f.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_void_p,
                  C.POINTER(C.c_int32), C.c_void_p]
    pc = p.to_c()
    sm = None if smask_ext is None else np.ascontiguousarray(smask_ext, np.int8)
    mp = None if marcap_ext is None else np.ascontiguousarray(marcap_ext, np.int32)
    rq = None if reqp is None else _f32(reqp)
    # capacity guard: the oracle writes at most nvoid_max cubes
    pc.nvoid_max = min(p.nvoid_max, cap)
    st = f(C.byref(pc), ptr(u1, C.c_float), ptr(dv, C.c_float),
           None if sm is None else sm.ctypes.data, None if mp is None else mp.ctypes.data,
           None if rq is None else rq.ctypes.data, C.byref(cubes.c), C.byref(nvoid),
           flags.ctypes.data, C.byref(nc), order.ctypes.data)
    if st == 4 and cap < p.nvoid_max:
        raise OracleError("oracle cube buffer too small for this test grid")
    _chk(st)
    return dict(cubes=cubes.view(nvoid.value), nvoid=nvoid.value, flags=flags,
                ncand=nc.value, order=order[:nc.value].copy())


def indexx(arr):
    arr = _f32(arr)
    out = np.zeros(len(arr), np.int32)
    f = lib().orc_indexx
    f.argtypes = [C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_int32)]
    _chk(f(len(arr), ptr(arr, C.c_float), ptr(out, C.c_int32)))
    return out


def merge_post(p: Params, nvoid, cubes: dict, u1co_ext, meandens):
    g, _ = grid_setup(p)
    cb = Cubes.from_dict(cubes, nvoid)
    vo = Voids(nvoid, g.ne)
    f = lib().orc_merge_post
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_float), C.c_float, C.c_void_p]
    pc = p.to_c()
    _chk(f(C.byref(pc), nvoid, C.byref(cb.c), ptr(_f32(u1co_ext), C.c_float),
           C.c_float(meandens), C.byref(vo.c)))
    return vo.view(nvoid)


def run_level(p: Params, parts: dict):
    """particles -> catalogue on the CPU (a5-a24)."""
    g, _ = grid_setup(p)
    pg = particles_to_grid(p, *(parts.get(k) for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
    u1, dv, md = fields(p, pg["u_mass"], pg["u2"], pg["u3"], pg["u4"])
    vf = voidfind(p, u1, dv)
    cat = merge_post(p, vf["nvoid"], vf["cubes"], u1, md)
    return dict(grid=pg, u1co=u1, diverco=dv, meandens=md, vf=vf, cat=cat)


def next_level(p: Params, nvoid, marca_ext, uvoid, req):
    """Parent map and radii of the next level (numpy restatement).

    MARCAP(2NX)^3 = MARCA(INT((IX-1)/2.)+1, ...) and REQP(IND) = REQ(IND) for
    main voids (src/avism.f90:2123-2157), then MARCAP2 = MARCAP on 1..2NX with
    the periodic ghost shell of INT_MAKE_PERIODIC (src/avism.f90:1670-1674,
    src/num.f90:137-181).  Returns (MARCAP2 flattened x-fastest, REQP)."""
    g, _ = grid_setup(p)
    pn = Params(**{**p.__dict__, "nx": 2 * p.nx, "level": p.level + 1})
    gn, _ = grid_setup(pn)
    ne, nx = g.ne, g.nx
    m = np.asarray(marca_ext, np.int32).reshape(ne, ne, ne)          # [k][j][i]
    lo = 1 - g.low1                                                   # offset of inner cell 1
    inner = m[lo:lo + nx, lo:lo + nx, lo:lo + nx]
    fine = inner.repeat(2, 0).repeat(2, 1).repeat(2, 2)                # MARCAP(2NX)^3
    nx2 = 2 * nx
    idx = (np.arange(gn.low1, gn.low2 + 1) - 1) % nx2                  # periodic ghost fill
    ext = fine[np.ix_(idx, idx, idx)]
    uv = np.asarray(uvoid, np.int32)[:nvoid]
    rq = np.where(uv == -1, np.asarray(req, np.float32)[:nvoid], np.float32(0.0)).astype(np.float32)
    return np.ascontiguousarray(ext).ravel(), rq


def run_sublevel(p: Params, parts: dict, marcap_ext, reqp):
    """A level below the first: particles -> catalogue with the parent map."""
    pg = particles_to_grid(p, *(parts.get(k) for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
    u1, dv, md = fields(p, pg["u_mass"], pg["u2"], pg["u3"], pg["u4"])
    vf = voidfind(p, u1, dv, marcap_ext=marcap_ext, reqp=reqp)
    cat = merge_post(p, vf["nvoid"], vf["cubes"], u1, md)
    return dict(u1co=u1, diverco=dv, meandens=md, vf=vf, cat=cat)

