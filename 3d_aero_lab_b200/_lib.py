"""Loader and ctypes prototypes of libaero3d.so (the C ABI of include/aero3d.h).

There is no fallback: if the library is missing or fails to load, importing the solver
raises.  Every call goes through `check()`, which turns a non-zero status into
`AeroError` carrying the library's own message (a3d_last_error).
"""
import ctypes as C
import os

import numpy as np

from .abi import STATUS_NAMES, a3d_request, a3d_result, a3d_server_config, a3d_shape

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaero3d.so")


class AeroError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_sp = C.POINTER(a3d_shape)

PROTOS = {
    "a3d_last_error": (C.c_char_p, []),
    "a3d_abi_version": (C.c_int, []),
    "a3d_grid_build": (C.c_int, [_sp, C.c_double, C.c_int32, _dp, _dp, _dp, _i32, C.POINTER(C.c_double), _dp]),
    "a3d_geom_build": (C.c_int, [_sp, _i32, _dp, _dp, _dp, C.c_double, C.c_double, _u8, _fp, _fp, _fp, _fp, _fp,
                                 _i64, _i32]),
    "a3d_solver_force_list": (C.c_int, [_vp, C.POINTER(C.c_int64), C.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "a3d_solver_create": (C.c_int, [_i32, _dp, _dp, _dp, _u8, _fp, _fp, _fp, _fp, _fp, C.c_int, C.POINTER(_vp)]),
    "a3d_solver_create_shape": (C.c_int, [_sp, _i32, _dp, _dp, _dp, C.c_double, C.c_double, C.c_int,
                                          C.POINTER(_vp)]),
    "a3d_solver_destroy": (C.c_int, [_vp]),
    "a3d_solver_dims": (C.c_int, [_vp, _i32, C.POINTER(C.c_int64)]),
    "a3d_solver_set_opt": (C.c_int, [_vp, C.c_double, C.c_int32]),
    "a3d_solver_set_free": (C.c_int, [_vp, _dp]),
    "a3d_solver_set_fix": (C.c_int, [_vp, _dp]),
    "a3d_solver_reset": (C.c_int, [_vp]),
    "a3d_solver_step": (C.c_int, [_vp, C.c_int32]),
    "a3d_solver_iterations": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "a3d_solver_read": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "a3d_solver_write": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "a3d_solver_forces": (C.c_int, [_vp] + [C.c_double] * 6 + [_dp]),
    "a3d_solver_trefftz": (C.c_int, [_vp] + [C.c_double] * 4 + [C.POINTER(C.c_double)]),
    "a3d_solver_residual": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_double)]),
    "a3d_solver_mach_max": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_double)]),
    "a3d_solver_set_kernel": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "a3d_solver_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "a3d_solver_sample": (C.c_int, [_vp, C.c_int32, _dp, _dp, _i32]),
    "a3d_solver_interp_state": (C.c_int, [_vp, _vp]),
    "a3d_solver_sync": (C.c_int, [_vp]),
    "a3d_solver_create_shape_slab": (C.c_int, [_sp, _i32, _dp, _dp, _dp, C.c_double, C.c_double,
                                               C.c_int32, C.c_int32, C.c_int, C.POINTER(_vp)]),
    "a3d_solver_set_owned": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "a3d_solver_stage": (C.c_int, [_vp, C.c_int32]),
    "a3d_solver_copy_planes": (C.c_int, [_vp, C.c_int32, _vp, C.c_int32, C.c_int32, C.c_int32]),
    "a3d_solver_plane_ptr": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(_vp),
                                       C.POINTER(C.c_int64)]),
    "a3d_solver_residual_parts": (C.c_int, [_vp, _dp]),
    "a3d_solver_set_neighbors": (C.c_int, [_vp, _vp, _vp]),
    "a3d_solver_set_chunks": (C.c_int, [_vp, C.c_int32]),
    "a3d_solver_read_dt": (C.c_int, [_vp, C.c_void_p]),
    "a3d_solver_get_kernel": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "a3d_solver_set_wait_limit": (C.c_int, [_vp, C.c_uint32]),
    "a3d_solver_get_chunks": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "a3d_solver_sync_neighbors": (C.c_int, [_vp]),
    "a3d_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int32, C.POINTER(_vp)]),
    "a3d_batch_destroy": (C.c_int, [_vp]),
    "a3d_batch_step": (C.c_int, [_vp, C.c_int32]),
    "a3d_batch_sync": (C.c_int, [_vp]),
    "a3d_batch_set_schedule": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "a3d_batch_set_mode": (C.c_int, [_vp, C.c_int32]),
    "a3d_batch_get_mode": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "a3d_batch_get_schedule": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "a3d_batch_tune": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_float)]),
    "a3d_server_create": (C.c_int, [C.POINTER(a3d_server_config), C.POINTER(_vp)]),
    "a3d_server_submit": (C.c_int, [_vp, C.POINTER(a3d_request), C.POINTER(C.c_int64)]),
    "a3d_server_poll": (C.c_int, [_vp, C.c_int64, C.POINTER(a3d_result), C.POINTER(C.c_int32)]),
    "a3d_server_wait": (C.c_int, [_vp, C.c_int64, C.c_double, C.POINTER(a3d_result)]),
    "a3d_server_stats": (C.c_int, [_vp, _i64]),
    "a3d_server_destroy": (C.c_int, [_vp]),
    "a3d_forces_noalloc": (C.c_int, [_vp] * 5 + [C.c_int64] + [_vp] * 5 + [C.c_double] * 6 + [_vp, _dp]),
}

_lib = None


def lib():
    """Load libaero3d.so (building it first if it is absent and nvcc is available)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise AeroError(status, lib().a3d_last_error().decode(errors="replace"))
    return status


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)
