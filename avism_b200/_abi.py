"""ctypes mirror of the C-ABI structs in include/avism_gpu.h.

The structs are plain C: avism_params mirrors config/voids.dat (read by the
reference at src/avism.f90:173-254), avism_cubes holds the cube arrays VOIDFIND
leaves in module COMMONDATA (src/commondata.f90:104-110), avism_voids the arrays
of src/avism.f90:1758-1773.  Helper classes own numpy buffers and hand out the
pointer structs the C functions fill.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

# status codes (include/avism_gpu.h)
AVISM_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_OOM", 4: "ERR_NVOID_MAX",
    5: "ERR_OUT_OF_BOX", 6: "ERR_TIMEOUT", 7: "ERR_NO_DEVICE", 8: "ERR_UNSUPPORTED",
    9: "ERR_INTERNAL", 10: "ERR_IO",
}
# messages of the reference's STOP statements for the codes that have one
STOP_TEXT = {
    4: "NVOID > NVOID_MAX!! Increase NVOID_MAX",            # src/voidfinding.f90:467-470
    5: "Particles outside the bounding box! Check L0!",       # src/avism.f90:580-586
}

UM = np.float32(9.1717e18)      # MASCLET mass unit [Msun]   (src/commondata.f90:19)
UV = np.float32(299792.458)     # velocity unit [km/s]       (src/commondata.f90:18)
UL = np.float32(10.98)          # length unit [Mpc]          (src/commondata.f90:17)


class AvismParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("periodic", C.c_int32), ("lado0", C.c_float),
        ("ache", C.c_float), ("omega0", C.c_float), ("zeta", C.c_float),
        ("nvoid_max", C.c_int32), ("dens_thre", C.c_float), ("dens_thre2", C.c_float),
        ("grad_thre", C.c_float), ("div_thre", C.c_float), ("rmin", C.c_float),
        ("rmin_sub", C.c_float), ("kneighbours", C.c_int32),
        ("flag_vel_interp", C.c_int32), ("flag_dens_interp", C.c_int32),
        ("level", C.c_int32), ("levmin", C.c_int32), ("learned", C.c_int32),
        ("kernel_mode", C.c_int32), ("no_velocities", C.c_int32),
        ("flag_dens", C.c_int32), ("flag_div", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


class AvismPatchesC(C.Structure):
    """avism_patches: a MASCLET snapshot's level-1 patches."""
    _fields_ = ([("npatch", C.c_int32)] +
                [(n, C.POINTER(C.c_int32)) for n in ("nx", "ny", "nz", "ix", "iy", "iz")] +
                [(n, C.POINTER(C.c_float)) for n in ("rx", "ry", "rz")] +
                [("offset", C.POINTER(C.c_int64))] +
                [(n, C.POINTER(C.c_float)) for n in ("u11g", "u12g", "u13g", "u14g")])


def patches_c(amr: dict):
    """(AvismPatchesC, arrays to keep alive) of a dict with the patch sizes
    nx..nz, first base cells ix..iz, corners rx..rz, offsets (npatch + 1) and
    the cells u11g..u14g."""
    keep = {}
    for k in ("nx", "ny", "nz", "ix", "iy", "iz"):
        keep[k] = np.ascontiguousarray(amr[k], np.int32)
    for k in ("rx", "ry", "rz", "u11g", "u12g", "u13g", "u14g"):
        keep[k] = np.ascontiguousarray(amr[k], np.float32)
    keep["offset"] = np.ascontiguousarray(amr["offset"], np.int64)
    s = AvismPatchesC(npatch=len(keep["nx"]))
    for k, v in keep.items():
        ct = C.c_int32 if v.dtype == np.int32 else (C.c_int64 if v.dtype == np.int64 else C.c_float)
        setattr(s, k, v.ctypes.data_as(C.POINTER(ct)))
    return s, keep


class AvismGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("nplus", C.c_int32), ("low1", C.c_int32), ("low2", C.c_int32),
        ("ne", C.c_int32), ("rad_lo", C.c_int32), ("rad_hi", C.c_int32),
        ("dx", C.c_float), ("rx1", C.c_float), ("lado", C.c_float), ("lado0plus", C.c_float),
        ("rete", C.c_float), ("rote", C.c_float), ("hte", C.c_float),
    ]


_I32P = C.POINTER(C.c_int32)
_F32P = C.POINTER(C.c_float)


class AvismCubesC(C.Structure):
    _fields_ = [(n, _I32P) for n in (
        "inicio_x", "final_x", "inicio_y", "final_y", "inicio_z", "final_z",
        "icx", "icy", "icz", "father")] + [("vol", _F32P)] + [
        (n, _F32P) for n in ("rini_x", "rfin_x", "rini_y", "rfin_y", "rini_z", "rfin_z")]


class AvismVoidsC(C.Structure):
    _fields_ = [("indice", _I32P), ("uvoid", _I32P), ("ncellv", _I32P)] + [
        (n, _F32P) for n in ("volnew", "req", "xc", "yc", "zc", "gxc", "gyc", "gzc",
                             "eps", "ip", "umean", "mtot")] + [
        ("marca", _I32P), ("nvoid2", C.c_int32), ("nvoidt", C.c_int32),
        ("volt_clean", C.c_double)]


CUBE_INT = ("inicio_x", "final_x", "inicio_y", "final_y", "inicio_z", "final_z",
            "icx", "icy", "icz", "father")
CUBE_FLT = ("vol", "rini_x", "rfin_x", "rini_y", "rfin_y", "rini_z", "rfin_z")
VOID_INT = ("indice", "uvoid", "ncellv")
VOID_FLT = ("volnew", "req", "xc", "yc", "zc", "gxc", "gyc", "gzc", "eps", "ip",
            "umean", "mtot")


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Cubes:
    """numpy-owned cube arrays (capacity n) and their C pointer struct."""

    def __init__(self, n: int):
        n = max(int(n), 1)
        self.cap = n
        self.arr = {k: np.zeros(n, np.int32) for k in CUBE_INT}
        self.arr.update({k: np.zeros(n, np.float32) for k in CUBE_FLT})
        self.c = AvismCubesC(**{k: ptr(self.arr[k], C.c_int32) for k in CUBE_INT},
                             **{k: ptr(self.arr[k], C.c_float) for k in CUBE_FLT})

    def view(self, nvoid: int, copy: bool = True) -> dict:
        return {k: (v[:nvoid].copy() if copy else v[:nvoid]) for k, v in self.arr.items()}

    @classmethod
    def from_dict(cls, d: dict, nvoid: int) -> "Cubes":
        c = cls(nvoid)
        for k in CUBE_INT + CUBE_FLT:
            c.arr[k][:nvoid] = d[k][:nvoid]
        return c


class Voids:
    """numpy-owned catalogue arrays (nvoid entries + ext MARCA grid)."""

    def __init__(self, n: int, ne: int | None = None):
        n = max(int(n), 1)
        self.arr = {k: np.zeros(n, np.int32) for k in VOID_INT}
        self.arr.update({k: np.zeros(n, np.float32) for k in VOID_FLT})
        self.marca = np.zeros(ne ** 3, np.int32) if ne else None
        kw = {k: ptr(self.arr[k], C.c_int32) for k in VOID_INT}
        kw.update({k: ptr(self.arr[k], C.c_float) for k in VOID_FLT})
        kw["marca"] = ptr(self.marca, C.c_int32) if self.marca is not None else _I32P()
        self.c = AvismVoidsC(**kw)

    def view(self, nvoid: int, copy: bool = True) -> dict:
        d = {k: (v[:nvoid].copy() if copy else v[:nvoid]) for k, v in self.arr.items()}
        d["nvoid2"] = int(self.c.nvoid2)
        d["nvoidt"] = int(self.c.nvoidt)
        d["volt_clean"] = float(self.c.volt_clean)
        if self.marca is not None:
            d["marca"] = self.marca.copy() if copy else self.marca
        return d


@dataclass
class Params:
    """Python view of avism_params; defaults are the thresholds the AVISM
    project's own README recommends (its lines 209-224) with h=0.678,
    Omega_m=0.31 (config/voids.dat:12)."""
    nx: int = 64
    periodic: int = 1
    lado0: float = 100.0
    ache: float = 0.678
    omega0: float = 0.31
    zeta: float = 0.0
    nvoid_max: int = 30_000_000
    dens_thre: float = -0.8
    dens_thre2: float = 10.0
    grad_thre: float = 0.25
    div_thre: float = 0.0
    rmin: float = 3.0
    rmin_sub: float = 3.0
    kneighbours: int = 32
    flag_vel_interp: int = 1
    flag_dens_interp: int = 1
    level: int = 0
    levmin: int = 0
    learned: int = 0
    kernel_mode: int = 1
    no_velocities: int = 0
    flag_dens: int = 0
    flag_div: int = 0
    extra: dict = field(default_factory=dict)

    def to_c(self) -> AvismParams:
        p = AvismParams()
        for name, _ in AvismParams._fields_:
            if name == "reserved":
                continue
            setattr(p, name, getattr(self, name))
        return p
