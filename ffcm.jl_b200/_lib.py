"""ctypes binding of libffcm_b200.so (the C ABI declared in include/ffcm_b200.h).

The shared library is built in-tree by `ffcm.jl_b200/Makefile` (nvcc,
sm_100a). There is no fallback: if the library is missing, importing the
binding raises, so a machine without the built CUDA library fails loudly.
"""
from __future__ import annotations

import ctypes
import os
import re
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libffcm_b200.so"
HEADER = PKG_DIR.parent / "include" / "ffcm_b200.h"

# status codes (include/ffcm_b200.h)
OK = 0
ERR_ARGUMENT = 1
ERR_DIMENSION = 2
ERR_OOM = 3
ERR_CUDA = 4
ERR_TIMEOUT = 5
ERR_UNSUPPORTED = 6
ERR_STATE = 7

FLOAT32 = 0
FLOAT64 = 1

# conjugate gradients (ffcm_cg_solve)
CG_INITIAL_GUESS = 1
CG_STATUS = {1: "converged", 2: "maxiter", 3: "breakdown"}
HOST = 0
DEVICE = 1

FFT_PLANNING = {"estimate": 0, "measure": 1, "patient": 2}

# stencil arithmetic (ffcm_set_stencil)
STENCIL = {"reference": 0, "float64": 1}

BUF = dict(Y_WRAPPED=0, Y_SORTED=1, F_SORTED=2, CELL_HASH=3, ORIGINAL_INDEX=4, CELL_START=5,
           CELL_END=6, FORCE_DENSITY=7, FLUID_VELOCITY=8, K_X=9, K_Y=10, K_Z=11,
           NEIGHBOR_MAP=12)

STAGES = ["h2d", "cell_list", "spread", "fft_x_fwd", "fft_y_fwd", "fft_z_stokes", "fft_y_inv",
          "fft_x_inv", "interpolate", "correct", "d2h"]

_c = ctypes
_vp = _c.c_void_p
_i32 = _c.c_int32
_i64 = _c.c_int64
_d = _c.c_double
_dp = _c.POINTER(_c.c_double)
_i32p = _c.POINTER(_c.c_int32)
_i64p = _c.POINTER(_c.c_int64)

SIGNATURES = {
    "ffcm_last_error": (_c.c_char_p, []),
    "ffcm_version": (_c.c_int, []),
    "ffcm_validate_config": (_c.c_int, [_i32, _dp, _d, _i64, _d, _d, _i32p, _i32, _d, _i32, _i32]),
    "ffcm_derive_scalars": (_c.c_int, [_i32, _dp, _d, _d, _d, _i32p, _i32p, _dp, _dp, _dp, _dp,
                                       _dp, _dp]),
    "ffcm_create": (_c.c_int, [_c.POINTER(_vp), _i32, _dp, _d, _i64, _d, _d, _i32p, _i32, _d,
                               _i32, _i32, _i32]),
    "ffcm_destroy": (_c.c_int, [_vp]),
    "ffcm_get_info": (_c.c_int, [_vp, _i64p, _i32p, _i64p]),
    "ffcm_set_stencil": (_c.c_int, [_vp, _i32]),
    "ffcm_get_stencil": (_c.c_int, [_vp, _i32p]),
    "ffcm_get_tuning": (_c.c_int, [_vp, _i32p]),
    "ffcm_wisdom_export": (_i64, [_c.c_char_p, _i64]),
    "ffcm_wisdom_import": (_c.c_int, [_c.c_char_p]),
    "ffcm_mobility": (_c.c_int, [_vp, _vp, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _i32,
                                 _vp]),
    "ffcm_wrap_positions": (_c.c_int, [_vp, _vp, _i32, _vp]),
    "ffcm_assign_cells": (_c.c_int, [_vp, _vp]),
    "ffcm_sort_particles_by_cell": (_c.c_int, [_vp, _vp, _i32, _vp]),
    "ffcm_spread_forces": (_c.c_int, [_vp, _vp]),
    "ffcm_stokes_solve": (_c.c_int, [_vp, _vp]),
    "ffcm_interpolate_velocities": (_c.c_int, [_vp, _vp, _i32, _vp]),
    "ffcm_correct_velocities": (_c.c_int, [_vp, _vp, _i32, _vp]),
    "ffcm_buffer_bytes": (_i64, [_vp, _i32]),
    "ffcm_get_buffer": (_c.c_int, [_vp, _i32, _vp, _i64, _i32, _vp]),
    "ffcm_set_buffer": (_c.c_int, [_vp, _i32, _vp, _i64, _i32, _vp]),
    "ffcm_synchronize": (_c.c_int, [_vp, _vp]),
    "ffcm_profile_begin": (_c.c_int, [_vp]),
    "ffcm_profile_end": (_c.c_int, [_vp, _dp, _i64p]),
    "ffcm_launch_count": (_i64, [_vp]),
    "ffcm_batch_create": (_c.c_int, [_c.POINTER(_vp), _i32, _i64, _dp, _dp, _i64p, _d, _d, _i32p,
                                     _i32, _d, _i32, _i32]),
    "ffcm_batch_destroy": (_c.c_int, [_vp]),
    "ffcm_batch_mobility": (_c.c_int, [_vp, _vp, _vp, _vp, _i32, _vp]),
    "ffcm_batch_get_info": (_c.c_int, [_vp, _i64p, _i64p, _i32p, _i64p]),
    "ffcm_mobility_checkpoint": (_c.c_int, [_vp, _vp, _vp, _vp, _i32, _vp]),
    "ffcm_adjoint": (_c.c_int, [_vp, _vp, _vp, _vp, _i32, _vp]),
    "ffcm_objective_gradient": (_c.c_int, [_vp, _dp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "ffcm_sort_cells_noalloc": (_c.c_int, [_vp, _i64, _i32, _vp, _vp, _vp, _vp]),
    "ffcm_set_positions": (_c.c_int, [_vp, _vp, _i32, _vp]),
    "ffcm_mobility_apply": (_c.c_int, [_vp, _vp, _vp, _i32, _vp]),
    "ffcm_cg_solve": (_c.c_int, [_vp, _vp, _vp, _i32, _c.c_double, _c.c_double, _i32, _i32, _vp, _vp, _vp,
                                 _vp]),
    "ffcm_dist_partition": (_c.c_int, [_i32, _i32p, _i32, _i32, _i32p]),
    "ffcm_dist_create": (_c.c_int, [_c.POINTER(_vp), _i32, _dp, _d, _i64, _d, _d, _i32p, _i32, _d, _i32, _i32,
                                    _i32]),
    "ffcm_dist_buffers": (_c.c_int, [_vp, _c.POINTER(_vp), _c.POINTER(_vp), _i64p, _c.POINTER(_vp), _i32p]),
    "ffcm_dist_forward": (_c.c_int, [_vp, _vp, _vp, _i32, _vp]),
    "ffcm_dist_stokes": (_c.c_int, [_vp, _vp]),
    "ffcm_dist_interpolate": (_c.c_int, [_vp, _vp]),
    "ffcm_dist_correct": (_c.c_int, [_vp, _vp, _i32, _vp]),
}

_lib = None


def declared_symbols(header: Path = HEADER):
    """Names of every function declared in the public header."""
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ffcm_[a-z0-9_]+)\s*\(", text)))


def load(path: Path | None = None):
    """Load the built library (cached). Raises OSError if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("FFCM_B200_LIB", LIB_PATH))
    if not p.exists():
        raise OSError(f"libffcm_b200.so not built at {p}; run `make -C ffcm.jl_b200` "
                      "(or __graft_entry__.build())")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().ffcm_last_error()
    return msg.decode("utf-8", "replace") if msg else ""
