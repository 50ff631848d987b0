"""Host-side mirror of the reference's routines for the AVISM hot path.

Each method keeps the name of the Fortran routine it replaces and calls the
C-ABI of libavism_gpu.so (include/avism_gpu.h); arrays are numpy (host) or any
object exposing a CUDA device pointer through ``data_ptr()`` (torch tensors).
Errors raise AvismError carrying the status code and, where the reference
stops, its STOP text.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._abi import (AVISM_OK, STATUS_NAMES, STOP_TEXT, AvismGrid, Cubes, Params, Voids, ptr)


class AvismError(RuntimeError):
    def __init__(self, code: int, msg: str):
        self.code = code
        text = STOP_TEXT.get(code, "")
        super().__init__(f"avism status {code} ({STATUS_NAMES.get(code, '?')}): {msg}"
                         + (f" [{text}]" if text and text not in msg else ""))


def _vp(a):
    """void* of a numpy array (host) or a tensor-like with data_ptr() (device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return C.c_void_p(a.ctypes.data)
    raise TypeError(type(a))


def _f32(a):
    if hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=np.float32)


def grid_setup(p: Params):
    """MALLA (src/grid.f90:3-76) + the PBC extension (src/avism.f90:780-865)."""
    lib = _lib.load()
    g = AvismGrid()
    pc = p.to_c()
    st = lib.avism_gpu_grid_setup(C.byref(pc), C.byref(g), None)
    if st != AVISM_OK:
        raise AvismError(st, "grid setup")
    rad = np.zeros(g.rad_hi - g.rad_lo + 1, np.float32)
    lib.avism_gpu_grid_setup(C.byref(pc), C.byref(g), _vp(rad))
    return g, rad


# ---- on-disk formats (host only) ---------------------------------------------
def _io_chk(st, what):
    if st != AVISM_OK:
        raise AvismError(st, what)


def _path(p):
    return None if p is None else os.fsencode(p)


def read_particle_file(path) -> dict:
    """A READ_BINARY_PART_1 particle file (src/reader.f90:410-460): x, y, z, vx,
    vy, vz, m as stored (cMpc, km/s, Msun) and the redshift zeta."""
    lib = _lib.load()
    n, zeta = C.c_int64(), C.c_float()
    _io_chk(lib.avism_io_particle_header(_path(path), C.byref(n), C.byref(zeta)), f"particle file {path}")
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")
    out = {k: np.zeros(n.value, np.float32) for k in keys}
    _io_chk(lib.avism_io_read_particles(_path(path), n.value, *(_vp(out[k]) for k in keys)), f"particle file {path}")
    out["zeta"] = zeta.value
    return out


def read_particle_file_novel(path) -> dict:
    """A READ_BINARY_PART_2 particle file (src/reader.f90:465-519): x, y, z, m
    as stored, no velocities, and the redshift zeta."""
    lib = _lib.load()
    n, zeta = C.c_int64(), C.c_float()
    _io_chk(lib.avism_io_particle_header(_path(path), C.byref(n), C.byref(zeta)), f"particle file {path}")
    keys = ("x", "y", "z", "m")
    out = {k: np.zeros(n.value, np.float32) for k in keys}
    _io_chk(lib.avism_io_read_particles_novel(_path(path), n.value, *(_vp(out[k]) for k in keys)),
            f"particle file {path}")
    out["zeta"] = zeta.value
    return out


def read_grid_file(path, nx) -> dict:
    """A READ_BINARY_GRID file (src/reader.f90:523-552): the density contrast
    u1 and velocities u2..u4 (km/s) on nx^3 cells as stored, and zeta."""
    nc = int(nx) ** 3
    out = {k: np.zeros(nc, np.float32) for k in ("u1", "u2", "u3", "u4")}
    zeta = C.c_float()
    _io_chk(_lib.load().avism_io_read_grid(_path(path), int(nx), C.byref(zeta),
                                           *(_vp(out[k]) for k in ("u1", "u2", "u3", "u4"))), f"grid file {path}")
    out["zeta"] = zeta.value
    return out


def read_masclet_files(grid_path, gas_path, dm_path, nhy) -> dict:
    """A MASCLET snapshot (READ_MASCLET, src/reader.f90:86-405): the level-0 gas
    grids (u1g = delta + 1, u2g..u4g; nhy^3), every level's DM particles (x..m,
    level 0 first with mass MAP), and the header (nl, ndxyz0, zeta, map)."""
    lib = _lib.load()
    nl, nd0, zeta, mp = C.c_int32(), C.c_int32(), C.c_float(), C.c_float()
    n = C.c_int64()
    _io_chk(lib.avism_io_masclet_header(_path(grid_path), C.byref(nl), C.byref(nd0), C.byref(n), C.byref(zeta),
                                        C.byref(mp)), f"MASCLET grid file {grid_path}")
    nc = int(nhy) ** 3
    gas = {k: np.zeros(nc, np.float32) for k in ("u1g", "u2g", "u3g", "u4g")}
    parts = {k: np.zeros(max(n.value, 1), np.float32) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    got = C.c_int64()
    _io_chk(lib.avism_io_read_masclet(_path(grid_path), _path(gas_path), _path(dm_path), int(nhy),
                                      *(_vp(gas[k]) for k in ("u1g", "u2g", "u3g", "u4g")), n.value,
                                      *(_vp(parts[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
                                      C.byref(got)), f"MASCLET files {gas_path}, {dm_path}")
    parts = {k: v[:got.value] for k, v in parts.items()}
    out = dict(gas=gas, parts=parts, nl=nl.value, ndxyz0=nd0.value, zeta=zeta.value, map=mp.value)
    out["amr"] = read_masclet_patches(grid_path, gas_path, nhy) if nl.value >= 1 else None
    return out


def read_masclet_patches(grid_path, gas_path, nhy) -> dict:
    """The level-1 patches of a MASCLET snapshot (src/reader.f90:168-174,
    285-312, 393) as the `amr` argument of masclet_fields / run_level_masclet:
    nx..nz, ix..iz, rx..rz per patch, offset (npatch + 1) and the cells
    u11g (delta + 1), u12g, u13g, u14g."""
    lib = _lib.load()
    np_, nc = C.c_int32(), C.c_int64()
    _io_chk(lib.avism_io_masclet_patches_size(_path(grid_path), C.byref(np_), C.byref(nc)),
            f"MASCLET grid file {grid_path}")
    npatch, ncells = np_.value, nc.value
    out = {k: np.zeros(max(npatch, 1), np.int32) for k in ("nx", "ny", "nz", "ix", "iy", "iz")}
    out.update({k: np.zeros(max(npatch, 1), np.float32) for k in ("rx", "ry", "rz")})
    out["offset"] = np.zeros(npatch + 1, np.int64)
    out.update({k: np.zeros(max(ncells, 1), np.float32) for k in ("u11g", "u12g", "u13g", "u14g")})
    _io_chk(lib.avism_io_read_masclet_patches(
        _path(grid_path), _path(gas_path), int(nhy), npatch, ncells,
        *(_vp(out[k]) for k in ("nx", "ny", "nz", "ix", "iy", "iz", "rx", "ry", "rz", "offset",
                                "u11g", "u12g", "u13g", "u14g"))), f"MASCLET gas file {gas_path}")
    for k in ("nx", "ny", "nz", "ix", "iy", "iz", "rx", "ry", "rz"):
        out[k] = out[k][:npatch]
    for k in ("u11g", "u12g", "u13g", "u14g"):
        out[k] = out[k][:ncells]
    return out


def read_mask_file(path, ncox, nx):
    """The survey mask (src/avism.f90:403-418, 873-901) on the level's nx^3
    inner cells (int8) and (MASKLOW, MASKUPPER, MASKSIDE)."""
    sm = np.zeros(int(nx) ** 3, np.int8)
    lims = np.zeros(3, np.float32)
    _io_chk(_lib.load().avism_io_read_mask(_path(path), int(ncox), int(nx), _vp(sm), _vp(lims)), f"mask {path}")
    return sm, lims


def read_randoms_file(path) -> dict:
    """The survey randoms (src/avism.f90:1425-1444): x, y, z and weights w."""
    lib = _lib.load()
    n = C.c_int32()
    _io_chk(lib.avism_io_randoms_header(_path(path), C.byref(n)), f"randoms {path}")
    out = {k: np.zeros(n.value, np.float32) for k in ("x", "y", "z", "w")}
    _io_chk(lib.avism_io_read_randoms(_path(path), n.value, *(_vp(out[k]) for k in ("x", "y", "z", "w"))),
            f"randoms {path}")
    return out


def write_vel_cube(path, nx, u2, u3, u4):
    """vel_cube.dat (src/avism.f90:1198-1202): the three velocity grids raw."""
    _io_chk(_lib.load().avism_io_write_vel_cube(_path(path), int(nx), *(_vp(_f32(u)) for u in (u2, u3, u4))),
            f"vel_cube {path}")


def write_catalogue_headers(voids_path, cubes_path, nlev, levmin, levmax, ncox, ncoy, ncoz, lado0):
    """First lines of the voids (and cubes) files of one iteration (src/avism.f90:710-722)."""
    _io_chk(_lib.load().avism_io_write_headers(_path(voids_path), _path(cubes_path), nlev, levmin, levmax,
                                               ncox, ncoy, ncoz, lado0), "catalogue headers")


def append_catalogue_level(voids_path, p: Params, res: dict, nvoidp: int = 0, req_parent=None, cubes_path=None,
                           map_path=None, u1co_ext=None, diverco_ext=None):
    """One level of a run_level / run_sublevel result (``cubes``, ``nvoid``,
    ``cat``, ``meandens``) into the voids, cubes and map files
    (src/avism.f90:2026-2085)."""
    nv = int(res["nvoid"])
    cb = Cubes.from_dict(res["cubes"], nv) if res.get("cubes") is not None else None
    cat = res["cat"]
    vo = Voids(max(nv, 1), None)
    for k in vo.arr:
        vo.arr[k][:nv] = np.asarray(cat[k])[:nv]
    marca = cat.get("marca")
    if marca is not None:
        vo.marca = np.ascontiguousarray(marca, np.int32)
        vo.c.marca = ptr(vo.marca, C.c_int32)
    vo.c.nvoid2, vo.c.nvoidt, vo.c.volt_clean = int(cat["nvoid2"]), int(cat["nvoidt"]), float(cat["volt_clean"])
    rp = None if req_parent is None else _f32(req_parent)
    u1 = None if u1co_ext is None else _f32(u1co_ext)
    dv = None if diverco_ext is None else _f32(diverco_ext)
    pc = p.to_c()
    _io_chk(_lib.load().avism_io_append_level(
        _path(voids_path), _path(cubes_path), _path(map_path), C.byref(pc), nv, int(nvoidp),
        float(res["meandens"]), C.byref(cb.c) if cb else None, C.byref(vo.c), _vp(rp), _vp(u1), _vp(dv)),
        "catalogue level")


class AvismGPU:
    """One context on one GPU (avism_gpu_create)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.avism_gpu_create(C.byref(h), device)
        if st != AVISM_OK:
            raise AvismError(st, f"cannot open CUDA device {device} (sm_100 required)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.avism_gpu_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, st):
        if st != AVISM_OK:
            msg = self.lib.avism_gpu_last_error(self.h)
            raise AvismError(st, msg.decode() if msg else "")

    def stage_times(self):
        """{stage name: device ms} of the last call."""
        buf = (C.c_double * 64)()
        n = min(self.lib.avism_gpu_stage_times(self.h, buf, 64), 64)
        return {self.lib.avism_gpu_stage_name(self.h, i).decode() or f"s{i}": buf[i] for i in range(n)}

    def launches(self) -> int:
        return int(self.lib.avism_gpu_launches(self.h))

    # ---- warp-kNN counters (instrumentation, no reference counterpart) ---------
    def knn_counters(self, enable: bool = True) -> dict:
        """Counters of the last particles_to_grid / run_level call; enable
        turns collection on (or off) for the following calls."""
        out = np.zeros(9, np.int64)
        self._chk(self.lib.avism_gpu_knn_counters(self.h, int(enable), _vp(out), 9))
        keys = ("queries", "attempts", "scanned", "kept", "fallbacks", "exact_ranks", "ball_cells", "orphans",
                "norm0")
        return {k: int(out[i]) for i, k in enumerate(keys)}

    # ---- learned proposal (no reference counterpart) -----------------------------
    def proposal_load(self, params):
        params = _f32(params)
        self._chk(self.lib.avism_gpu_proposal_load(self.h, _vp(params), len(params)))

    def proposal_features(self, p: Params, parts: dict):
        """(features [nb^3, 12], nb, bin width) of the binning particles_to_grid uses."""
        a = {k: (_f32(parts[k]) if parts.get(k) is not None else None) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        nb, bw = C.c_int32(), C.c_float()
        pc = p.to_c()
        args = (self.h, C.byref(pc), len(a["x"]), *(_vp(a[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
        self._chk(self.lib.avism_gpu_proposal_features(*args, 0, None, C.byref(nb), C.byref(bw)))
        rows = nb.value ** 3
        feat = np.zeros((rows, 12), np.float32)
        self._chk(self.lib.avism_gpu_proposal_features(*args, rows, _vp(feat), C.byref(nb), C.byref(bw)))
        return feat, nb.value, bw.value

    def proposal_infer(self, feat, params):
        feat = np.ascontiguousarray(feat, np.float32)
        out = np.zeros((len(feat), 2), np.float32)
        self._chk(self.lib.avism_gpu_proposal_infer(self.h, len(feat), _vp(feat), _vp(_f32(params)), _vp(out)))
        return out

    def proposal_grad(self, feat, target, mask, params):
        feat = np.ascontiguousarray(feat, np.float32)
        g = np.zeros(len(params), np.float32)
        loss = C.c_float()
        self._chk(self.lib.avism_gpu_proposal_grad(self.h, len(feat), _vp(feat), _vp(_f32(target)), _vp(_f32(mask)),
                                                   _vp(_f32(params)), _vp(g), C.byref(loss)))
        return loss.value, g

    def proposal_train(self, feat, target, mask, params, steps, batch=4096, lr=1e-3, seed=0):
        feat = np.ascontiguousarray(feat, np.float32)
        prm = np.array(params, np.float32, copy=True)
        curve = np.zeros(max(steps, 1), np.float32)
        self._chk(self.lib.avism_gpu_proposal_train(self.h, len(feat), _vp(feat), _vp(_f32(target)), _vp(_f32(mask)),
                                                    steps, batch, lr, seed, _vp(prm), _vp(curve)))
        return prm, curve[:steps]

    # ---- kNN (knn_search, src/kdtree.f90:504-540) ----------------------------
    def knn_search(self, x, y, z, qx, qy, qz, k, box_l=0.0):
        x, y, z, qx, qy, qz = map(_f32, (x, y, z, qx, qy, qz))
        nq = len(qx)
        idx = np.zeros(nq * k, np.int64)
        dist = np.zeros(nq * k, np.float32)
        self._chk(self.lib.avism_gpu_knn(self.h, len(x), _vp(x), _vp(y), _vp(z), box_l, nq,
                                         _vp(qx), _vp(qy), _vp(qz), k, _vp(idx), _vp(dist)))
        return idx.reshape(nq, k), dist.reshape(nq, k)

    # ---- PPART_DENS / VVEL_INTERP_SPH_VW / FILL_H_ZEROS / DDENS_INTERP_SPH / TSC
    def particles_to_grid(self, p: Params, parts: dict, smask=None):
        a = {k: (_f32(parts[k]) if parts.get(k) is not None else None) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        n = len(a["x"])
        nc = p.nx ** 3
        out = [np.zeros(nc, np.float32) for _ in range(4)]
        h = np.zeros(n, np.float32)
        pd = np.zeros(n, np.float32)
        sm = None if smask is None else np.ascontiguousarray(smask, np.int8)
        pc = p.to_c()
        self._chk(self.lib.avism_gpu_particles_to_grid(
            self.h, C.byref(pc), n, *(_vp(a[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
            _vp(sm), *(_vp(o) for o in out), _vp(h), _vp(pd)))
        return dict(u_mass=out[0], u2=out[1], u3=out[2], u4=out[3], hpart=h, part_dens=pd)

    # ---- normalisation, DIVER_UNIFORM, REAL_MAKE_PERIODIC ---------------------
    def fields(self, p: Params, u_mass, u2, u3, u4):
        g, _ = grid_setup(p)
        ne3 = g.ne ** 3
        u1 = np.zeros(ne3, np.float32)
        dv = np.zeros(ne3, np.float32)
        md = C.c_float()
        pc = p.to_c()
        self._chk(self.lib.avism_gpu_fields(self.h, C.byref(pc),
                                            *(_vp(None if v is None else _f32(v)) for v in (u_mass, u2, u3, u4)),
                                            _vp(u1), _vp(dv), C.byref(md)))
        return u1, dv, md.value

    # ---- MARK_ALL + VOIDFIND --------------------------------------------------
    def voidfind(self, p: Params, u1co_ext, diverco_ext, smask_ext=None, marcap_ext=None, reqp=None,
                 capacity=None):
        g, _ = grid_setup(p)
        cap = int(capacity or min(p.nvoid_max, max(g.ne ** 3 // 8, 1024)))
        cubes = Cubes(cap)
        nv = C.c_int32()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        sm = None if smask_ext is None else np.ascontiguousarray(smask_ext, np.int8)
        mp = None if marcap_ext is None else np.ascontiguousarray(marcap_ext, np.int32)
        rq = None if reqp is None else _f32(reqp)
        self._chk(self.lib.avism_gpu_voidfind(self.h, C.byref(pc), _vp(_f32(u1co_ext)), _vp(_f32(diverco_ext)),
                                              _vp(sm), _vp(mp), _vp(rq), C.byref(cubes.c), C.byref(nv)))
        return cubes.view(nv.value), nv.value

    def mark_all(self, p: Params, u1co_ext, diverco_ext, smask_ext=None, marcap_ext=None):
        """MARK_ALL + the directional flag grids, one packed byte per ext cell."""
        g, _ = grid_setup(p)
        fl = np.zeros(g.ne ** 3, np.uint8)
        sm = None if smask_ext is None else np.ascontiguousarray(smask_ext, np.int8)
        mp = None if marcap_ext is None else np.ascontiguousarray(marcap_ext, np.int32)
        pc = p.to_c()
        self._chk(self.lib.avism_gpu_flags(self.h, C.byref(pc), _vp(_f32(u1co_ext)), _vp(_f32(diverco_ext)),
                                           _vp(sm), _vp(mp), _vp(fl)))
        return fl

    # ---- INDEXX (src/num.f90:2-84) --------------------------------------------
    def indexx(self, arr):
        arr = _f32(arr)
        out = np.zeros(len(arr), np.int32)
        self._chk(self.lib.avism_gpu_indexx(self.h, len(arr), _vp(arr), _vp(out)))
        return out

    # ---- MERGE_VOID + post-processing -----------------------------------------
    def merge_post(self, p: Params, nvoid, cubes: dict, u1co_ext, meandens, want_marca=True):
        g, _ = grid_setup(p)
        cb = Cubes.from_dict(cubes, nvoid)
        vo = Voids(nvoid, g.ne if want_marca else None)
        pc = p.to_c()
        self._chk(self.lib.avism_gpu_merge_post(self.h, C.byref(pc), nvoid, C.byref(cb.c),
                                                _vp(_f32(u1co_ext)), meandens, C.byref(vo.c)))
        return vo.view(nvoid)

    # ---- voids-in-voids (src/avism.f90:2123-2157, 1670-1674) --------------------
    def next_level(self, p: Params, nvoid, marca_ext, uvoid, req):
        """(MARCAP2 ext grid of the next level, REQP) from this level's catalogue."""
        pn = Params(**{**p.__dict__, "nx": 2 * p.nx, "level": p.level + 1})
        gn, _ = grid_setup(pn)
        out = np.zeros(gn.ne ** 3, np.int32)
        rq = np.zeros(max(nvoid, 1), np.float32)
        self._chk(self.lib.avism_gpu_next_level(self.h, C.byref(p.to_c()), nvoid,
                                                _vp(np.ascontiguousarray(marca_ext, np.int32)),
                                                _vp(np.ascontiguousarray(uvoid, np.int32)), _vp(_f32(req)),
                                                _vp(out), _vp(rq)))
        return out, rq[:nvoid]

    def run_sublevel(self, p: Params, parts: dict, marcap_ext, reqp, want_marca=False, capacity=None):
        g, _ = grid_setup(p)
        cap = int(capacity or p.nvoid_max)
        a = {k: (_f32(parts[k]) if parts.get(k) is not None else None) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        cubes = Cubes(cap)
        vo = Voids(cap, g.ne if want_marca else None)
        nv, md = C.c_int32(), C.c_float()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        rq = _f32(reqp)
        self._chk(self.lib.avism_gpu_run_sublevel(
            self.h, C.byref(pc), len(a["x"]), *(_vp(a[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
            _vp(np.ascontiguousarray(marcap_ext, np.int32)), _vp(rq), len(rq), C.byref(cubes.c), C.byref(nv),
            C.byref(vo.c), C.byref(md)))
        return dict(cubes=cubes.view(nv.value), nvoid=nv.value, cat=vo.view(nv.value), meandens=md.value)

    # ---- grid input (FLAG_DATA = 2, src/avism.f90:1316-1362) --------------------------
    def grid_fields(self, p: Params, nhy, u1g, u2g, u3g, u4g):
        """(U1CO ext, DIVERCO ext, MEANDENS) of the level from the input grids
        (U1G = delta + 1, velocities / UV, nhy^3)."""
        g, _ = grid_setup(p)
        u1 = np.zeros(g.ne ** 3, np.float32)
        dv = np.zeros(g.ne ** 3, np.float32)
        md = C.c_float()
        pc = p.to_c()
        self._chk(self.lib.avism_gpu_grid_fields(self.h, C.byref(pc), int(nhy),
                                                 *(_vp(_f32(a)) for a in (u1g, u2g, u3g, u4g)), _vp(u1), _vp(dv),
                                                 C.byref(md)))
        return u1, dv, md.value

    def run_level_grid(self, p: Params, nhy, u1g, u2g, u3g, u4g, want_marca=False, capacity=None):
        g, _ = grid_setup(p)
        cap = int(capacity or p.nvoid_max)
        cubes = Cubes(cap)
        vo = Voids(cap, g.ne if want_marca else None)
        nv, md = C.c_int32(), C.c_float()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        self._chk(self.lib.avism_gpu_run_level_grid(self.h, C.byref(pc), int(nhy),
                                                    *(_vp(_f32(a)) for a in (u1g, u2g, u3g, u4g)),
                                                    C.byref(cubes.c), C.byref(nv), C.byref(vo.c), C.byref(md)))
        return dict(cubes=cubes.view(nv.value), nvoid=nv.value, cat=vo.view(nv.value), meandens=md.value)

    # ---- MASCLET input (FLAG_DATA = 0) at levels <= 0 (src/avism.f90:980-1156) ------
    def _masclet_args(self, nhy, gas, parts, amr=None):
        """gas: (u1g = 1 + delta, u2g, u3g, u4g) at nhy^3 (velocity grids may be
        None when params.flag_div is 1 or -1 below level 1); parts: the DM
        particles or None; amr: the level-1 patches (a dict, see patches_c)."""
        from ._abi import patches_c
        pc_amr, keep_amr = patches_c(amr) if amr is not None else (None, None)
        g = tuple(None if a is None else _f32(a) for a in gas)
        if parts is None:
            a = {k: None for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
            n = 0
        else:
            a = {k: (_f32(parts[k]) if parts.get(k) is not None else None)
                 for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
            n = len(a["x"])
        args = (int(nhy), *(_vp(x) for x in g), C.byref(pc_amr) if pc_amr is not None else None, n,
                *(_vp(a[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
        return args, (g, a, pc_amr, keep_amr)

    def masclet_fields(self, p: Params, nhy, gas, parts=None, amr=None):
        """(U1CO ext, DIVERCO ext, MEANDENS) of a MASCLET snapshot's level."""
        gr, _ = grid_setup(p)
        u1 = np.zeros(gr.ne ** 3, np.float32)
        dv = np.zeros(gr.ne ** 3, np.float32)
        md = C.c_float()
        pc = p.to_c()
        args, _keep = self._masclet_args(nhy, gas, parts, amr)
        self._chk(self.lib.avism_gpu_masclet_fields(self.h, C.byref(pc), *args, _vp(u1), _vp(dv), C.byref(md)))
        return u1, dv, md.value

    def run_level_masclet(self, p: Params, nhy, gas, parts=None, amr=None, want_marca=False, capacity=None):
        gr, _ = grid_setup(p)
        cap = int(capacity or p.nvoid_max)
        cubes = Cubes(cap)
        vo = Voids(cap, gr.ne if want_marca else None)
        nv, md = C.c_int32(), C.c_float()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        args, _keep = self._masclet_args(nhy, gas, parts, amr)
        self._chk(self.lib.avism_gpu_run_level_masclet(self.h, C.byref(pc), *args, C.byref(cubes.c), C.byref(nv),
                                                       C.byref(vo.c), C.byref(md)))
        return dict(cubes=cubes.view(nv.value), nvoid=nv.value, cat=vo.view(nv.value), meandens=md.value)

    def run_sublevel_masclet(self, p: Params, nhy, gas, marcap_ext, reqp, parts=None, amr=None, want_marca=False,
                             capacity=None):
        """A MASCLET level inside the parent voids (MARCAP2 and REQP of next_level)."""
        gr, _ = grid_setup(p)
        cap = int(capacity or p.nvoid_max)
        cubes = Cubes(cap)
        vo = Voids(cap, gr.ne if want_marca else None)
        nv, md = C.c_int32(), C.c_float()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        args, _keep = self._masclet_args(nhy, gas, parts, amr)
        mp = np.ascontiguousarray(marcap_ext, np.int32)
        rq = _f32(reqp)
        self._chk(self.lib.avism_gpu_run_sublevel_masclet(self.h, C.byref(pc), *args, _vp(mp), _vp(rq), len(rq),
                                                          C.byref(cubes.c), C.byref(nv), C.byref(vo.c),
                                                          C.byref(md)))
        return dict(cubes=cubes.view(nv.value), nvoid=nv.value, cat=vo.view(nv.value), meandens=md.value)

    # ---- survey mode (src/avism.f90:1420-1596) -------------------------------------
    def _survey_args(self, parts, rands, smask):
        a = {k: (_f32(parts[k]) if parts.get(k) is not None else None)
             for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        r = {k: _f32(rands[k]) for k in ("x", "y", "z", "w")}
        sm = np.ascontiguousarray(smask, np.int8)
        return (len(a["x"]), *(_vp(a[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")), len(r["x"]),
                *(_vp(r[k]) for k in ("x", "y", "z", "w")), _vp(sm)), sm

    def survey_fields(self, p: Params, parts: dict, rands: dict, smask):
        """(U1CO ext, DIVERCO ext, MEANDENS, the randoms' grid) in survey mode."""
        g, _ = grid_setup(p)
        u1 = np.zeros(g.ne ** 3, np.float32)
        dv = np.zeros(g.ne ** 3, np.float32)
        ur = np.zeros(p.nx ** 3, np.float32)
        md = C.c_float()
        args, _keep = self._survey_args(parts, rands, smask)
        pc = p.to_c()
        self._chk(self.lib.avism_gpu_survey_fields(self.h, C.byref(pc), *args, _vp(u1), _vp(dv), C.byref(md),
                                                   _vp(ur)))
        return u1, dv, md.value, ur

    def run_level_survey(self, p: Params, parts: dict, rands: dict, smask, want_marca=False, capacity=None):
        g, _ = grid_setup(p)
        cap = int(capacity or p.nvoid_max)
        cubes = Cubes(cap)
        vo = Voids(cap, g.ne if want_marca else None)
        nv, md = C.c_int32(), C.c_float()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        args, _keep = self._survey_args(parts, rands, smask)
        self._chk(self.lib.avism_gpu_run_level_survey(self.h, C.byref(pc), *args, C.byref(cubes.c), C.byref(nv),
                                                      C.byref(vo.c), C.byref(md)))
        return dict(cubes=cubes.view(nv.value), nvoid=nv.value, cat=vo.view(nv.value), meandens=md.value)

    # ---- whole level ------------------------------------------------------------
    @staticmethod
    def level_buffers(p: Params, capacity=None, want_marca=False):
        """Caller-owned cube and catalogue arrays for run_level(bufs=...), reused
        across calls the way the Fortran driver keeps its COMMONDATA arrays."""
        g, _ = grid_setup(p)
        cap = int(capacity or p.nvoid_max)
        return Cubes(cap), Voids(cap, g.ne if want_marca else None)

    def run_level(self, p: Params, parts: dict, want_marca=False, want_cubes=True, capacity=None, bufs=None):
        """One level, particles -> catalogue.  With bufs (from level_buffers) the
        results are views of those arrays, valid until their next use."""
        g, _ = grid_setup(p)
        a = {k: (_f32(parts[k]) if parts.get(k) is not None else None) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        n = len(a["x"])
        if bufs is not None:
            cubes, vo = bufs
            cap = min(cubes.cap, len(vo.arr["indice"]))
            if want_marca and vo.marca is None:
                raise ValueError("run_level: want_marca needs buffers made with want_marca=True")
        else:
            cap = int(capacity or p.nvoid_max)
            cubes = Cubes(cap) if want_cubes else None
            vo = Voids(cap, g.ne if want_marca else None)
        nv = C.c_int32()
        md = C.c_float()
        pc = p.to_c()
        pc.nvoid_max = min(p.nvoid_max, cap)
        self._chk(self.lib.avism_gpu_run_level(
            self.h, C.byref(pc), n, *(_vp(a[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
            C.byref(cubes.c) if cubes else None, C.byref(nv), C.byref(vo.c), C.byref(md)))
        cp = bufs is None
        return dict(cubes=cubes.view(nv.value, cp) if cubes else None, nvoid=nv.value,
                    cat=vo.view(nv.value, cp), meandens=md.value)
