"""Loads libavism_gpu.so (the C-ABI of include/avism_gpu.h) and declares its
entry points.  There is no fallback: without the library or a B200 the calls
raise."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libavism_gpu.so")

_c_void = C.c_void_p
_i32, _i64, _f32 = C.c_int32, C.c_int64, C.c_float

# name -> (restype, argtypes); pointers are passed as void* (host or device)
SIGNATURES = {
    "avism_gpu_create": (C.c_int, [C.POINTER(_c_void), C.c_int]),
    "avism_gpu_destroy": (C.c_int, [_c_void]),
    "avism_gpu_last_error": (C.c_char_p, [_c_void]),
    "avism_gpu_stage_times": (C.c_int, [_c_void, _c_void, C.c_int]),
    "avism_gpu_stage_name": (C.c_char_p, [_c_void, C.c_int]),
    "avism_gpu_launches": (C.c_int64, [_c_void]),
    "avism_gpu_grid_setup": (C.c_int, [_c_void, _c_void, _c_void]),
    "avism_gpu_knn": (C.c_int, [_c_void, _i64, _c_void, _c_void, _c_void, _f32, _i64,
                                _c_void, _c_void, _c_void, _i32, _c_void, _c_void]),
    "avism_gpu_particles_to_grid": (C.c_int, [_c_void, _c_void, _i64] + [_c_void] * 14),
    "avism_gpu_fields": (C.c_int, [_c_void, _c_void] + [_c_void] * 7),
    "avism_gpu_voidfind": (C.c_int, [_c_void, _c_void] + [_c_void] * 7),
    "avism_gpu_flags": (C.c_int, [_c_void, _c_void] + [_c_void] * 5),
    "avism_gpu_indexx": (C.c_int, [_c_void, _i32, _c_void, _c_void]),
    "avism_gpu_merge_post": (C.c_int, [_c_void, _c_void, _i32, _c_void, _c_void, _f32, _c_void]),
    "avism_gpu_run_level": (C.c_int, [_c_void, _c_void, _i64] + [_c_void] * 7 + [_c_void] * 4),
    "avism_gpu_knn_counters": (C.c_int, [_c_void, C.c_int, _c_void, C.c_int]),
    "avism_gpu_proposal_load": (C.c_int, [_c_void, _c_void, _i32]),
    "avism_gpu_proposal_features": (C.c_int, [_c_void, _c_void, _i64] + [_c_void] * 7 + [_i64, _c_void, _c_void,
                                                                                       _c_void]),
    "avism_gpu_proposal_infer": (C.c_int, [_c_void, _i64, _c_void, _c_void, _c_void]),
    "avism_gpu_proposal_grad": (C.c_int, [_c_void, _i64] + [_c_void] * 6),
    "avism_gpu_proposal_train": (C.c_int, [_c_void, _i64, _c_void, _c_void, _c_void, _i32, _i32, _f32,
                                           C.c_uint32, _c_void, _c_void]),
    "avism_gpu_next_level": (C.c_int, [_c_void, _c_void, _i32] + [_c_void] * 5),
    "avism_gpu_run_sublevel": (C.c_int, [_c_void, _c_void, _i64] + [_c_void] * 9 + [_i32] + [_c_void] * 4),
    "avism_gpu_grid_fields": (C.c_int, [_c_void, _c_void, _i32] + [_c_void] * 7),
    "avism_gpu_run_level_grid": (C.c_int, [_c_void, _c_void, _i32] + [_c_void] * 8),
    "avism_gpu_masclet_fields": (C.c_int, [_c_void, _c_void, _i32] + [_c_void] * 5 + [_i64] + [_c_void] * 10),
    "avism_gpu_run_level_masclet": (C.c_int, [_c_void, _c_void, _i32] + [_c_void] * 5 + [_i64] + [_c_void] * 11),
    "avism_gpu_run_sublevel_masclet": (C.c_int, [_c_void, _c_void, _i32] + [_c_void] * 5 + [_i64] + [_c_void] * 9 +
                                       [_i32] + [_c_void] * 4),
    "avism_gpu_survey_fields": (C.c_int, [_c_void, _c_void, _i64] + [_c_void] * 7 + [_i64] + [_c_void] * 9),
    "avism_gpu_run_level_survey": (C.c_int, [_c_void, _c_void, _i64] + [_c_void] * 7 + [_i64] + [_c_void] * 9),
    "avism_gpu_knn_noalloc": (C.c_int, [C.c_int, _c_void, _i64, _c_void, _c_void, _c_void, _f32, _i64,
                                        _c_void, _c_void, _c_void, _i32, _c_void, _c_void, C.c_char_p,
                                        _i32]),
    "avism_io_particle_header": (C.c_int, [C.c_char_p, _c_void, _c_void]),
    "avism_io_read_particles": (C.c_int, [C.c_char_p, _i64] + [_c_void] * 7),
    "avism_io_read_particles_novel": (C.c_int, [C.c_char_p, _i64] + [_c_void] * 4),
    "avism_io_read_grid": (C.c_int, [C.c_char_p, _i32] + [_c_void] * 5),
    "avism_io_masclet_header": (C.c_int, [C.c_char_p, _c_void, _c_void, _c_void, _c_void, _c_void]),
    "avism_io_read_masclet": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, _i32] + [_c_void] * 4 + [_i64] +
                              [_c_void] * 8),
    "avism_io_masclet_patches_size": (C.c_int, [C.c_char_p, _c_void, _c_void]),
    "avism_io_read_masclet_patches": (C.c_int, [C.c_char_p, C.c_char_p, _i32, _i32, _i64] + [_c_void] * 14),
    "avism_io_read_mask": (C.c_int, [C.c_char_p, _i32, _i32, _c_void, _c_void]),
    "avism_io_randoms_header": (C.c_int, [C.c_char_p, _c_void]),
    "avism_io_read_randoms": (C.c_int, [C.c_char_p, _i32] + [_c_void] * 4),
    "avism_io_write_vel_cube": (C.c_int, [C.c_char_p, _i32] + [_c_void] * 3),
    "avism_io_write_headers": (C.c_int, [C.c_char_p, C.c_char_p] + [_i32] * 6 + [_f32]),
    "avism_io_append_level": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, _c_void, _i32, _i32, _f32]
                              + [_c_void] * 5),
}

_lib = None


def load(path: str | None = None):
    """Load the library; raises OSError if it has not been built."""
    global _lib
    if _lib is None:
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise OSError(f"{p} not built: run __graft_entry__.build() or python avism_b200/build.py")
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib
