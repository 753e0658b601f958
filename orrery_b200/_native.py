"""Loads the native library and declares the C ABI of include/orrery_lbm.h.

The library is the only implementation of the solvers: there is no Python or
CPU fallback.  If it is missing it is built in-tree (nvcc is part of the
toolchain); if that fails, importing the solvers raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import abi

_LOCK = threading.Lock()
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p
_st = ctypes.c_int32
_c3 = ctypes.POINTER(abi.CLbm3DConfig)
_c2 = ctypes.POINTER(abi.CLbm2DConfig)
_opt = ctypes.POINTER(abi.CSolverOptions)

# Every entry point of include/orrery_lbm.h: name -> (restype, argtypes).
SIGNATURES = {
    "orr_last_error": (ctypes.c_char_p, []),
    "orr_version": (ctypes.c_char_p, []),
    "orr_device_count": (_st, [_i32p]),
    "orr_lbm3d_validate": (_st, [_c3, _u8p, _dp, _opt, ctypes.c_char_p, ctypes.c_size_t]),
    "orr_lbm3d_create": (_st, [_c3, _u8p, _dp, _opt, ctypes.POINTER(_vp)]),
    "orr_lbm3d_destroy": (None, [_vp]),
    "orr_lbm3d_last_error": (ctypes.c_char_p, [_vp]),
    "orr_lbm3d_initialize": (_st, [_vp, _dp, _dp, _dp, _dp]),
    "orr_lbm3d_step": (_st, [_vp, ctypes.c_uint64]),
    "orr_lbm3d_steps": (_st, [_vp, _u64p]),
    "orr_lbm3d_set_inlet_velocity": (_st, [_vp, _dp]),
    "orr_lbm3d_inlet_velocity": (_st, [_vp, _dp]),
    "orr_lbm3d_force": (_st, [_vp, _dp]),
    "orr_lbm3d_macroscopic": (_st, [_vp, _dp, _dp, _dp, _dp]),
    "orr_lbm3d_populations": (_st, [_vp, _dp]),
    "orr_lbm3d_mass": (_st, [_vp, _dp]),
    "orr_lbm3d_link_count": (_st, [_vp, _u64p]),
    "orr_lbm3d_links": (_st, [_vp, _u32p, _u32p, _dp]),
    "orr_lbm3d_memory_bytes": (_st, [_c3, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, _u64p]),
    "orr_lbm3d_plan": (_st, [_c3, _u8p, _dp, _u64p, _u64p, _u64p, _u32p, _u32p, _dp]),
    "orr_lbm3d_node_counts": (_st, [_vp, _u64p, _u64p]),
    "orr_lbm3d_stream": (_st, [_vp, ctypes.POINTER(_vp)]),
    "orr_lbm3d_launch_count": (_st, [_vp, _u64p]),
    "orr_lbm3d_request_stall": (_st, [_vp, ctypes.c_uint32]),
    "orr_gl3d_buffer_slack": (ctypes.c_uint64, []),
    "orr_gl3d_create": (_st, [_vp, _u32p, ctypes.c_int32, ctypes.POINTER(_vp)]),
    "orr_gl3d_destroy": (None, [_vp]),
    "orr_gl3d_last_error": (ctypes.c_char_p, [_vp]),
    "orr_gl3d_step": (_st, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "orr_gl3d_moments": (_st, [_vp, _vp, _vp, _vp, _vp]),
    "orr_gl3d_link_force": (_st, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "orr_gl2d_create": (_st, [_vp, _u32p, ctypes.c_int32, ctypes.POINTER(_vp)]),
    "orr_gl2d_destroy": (None, [_vp]),
    "orr_gl2d_last_error": (ctypes.c_char_p, [_vp]),
    "orr_gl2d_step": (_st, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "orr_gl2d_moments": (_st, [_vp, _vp, _vp, _vp, _vp]),
    "orr_gl2d_link_force": (_st, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "orr_lbm3d_kernel_info": (_st, [_vp, ctypes.POINTER(abi.CKernelInfo)]),
    "orr_lbm3d_force_static": (_st, [ctypes.POINTER(abi.CForceLinks), _dp]),
    "orr_lbm2d_validate": (_st, [_c2, _u8p, _opt, ctypes.c_char_p, ctypes.c_size_t]),
    "orr_lbm2d_create": (_st, [_c2, _u8p, _opt, ctypes.POINTER(_vp)]),
    "orr_lbm2d_destroy": (None, [_vp]),
    "orr_lbm2d_last_error": (ctypes.c_char_p, [_vp]),
    "orr_lbm2d_initialize": (_st, [_vp, _dp, _dp, _dp]),
    "orr_lbm2d_step": (_st, [_vp, ctypes.c_uint64]),
    "orr_lbm2d_steps": (_st, [_vp, _u64p]),
    "orr_lbm2d_force": (_st, [_vp, _dp]),
    "orr_lbm2d_macroscopic": (_st, [_vp, _dp, _dp, _dp]),
    "orr_lbm2d_populations": (_st, [_vp, _dp]),
    "orr_lbm2d_mass": (_st, [_vp, _dp]),
    "orr_lbm2d_link_count": (_st, [_vp, _u64p]),
    "orr_lbm2d_links": (_st, [_vp, _u32p, _u32p]),
    "orr_lbm2d_stream": (_st, [_vp, ctypes.POINTER(_vp)]),
    "orr_lbm2d_launch_count": (_st, [_vp, _u64p]),
    "orr_batch3d_create": (_st, [ctypes.c_int32, ctypes.POINTER(_vp)]),
    "orr_batch3d_destroy": (None, [_vp]),
    "orr_batch3d_last_error": (ctypes.c_char_p, [_vp]),
    "orr_batch3d_add": (_st, [_vp, _vp]),
    "orr_batch3d_remove": (_st, [_vp, _vp]),
    "orr_batch3d_size": (_st, [_vp, _u32p, _u64p]),
    "orr_batch3d_set_schedule": (_st, [_vp, ctypes.POINTER(abi.CBatchSchedule)]),
    "orr_batch3d_schedule": (_st, [_vp, ctypes.POINTER(abi.CBatchSchedule)]),
    "orr_batch3d_step": (_st, [_vp, ctypes.c_uint64]),
    "orr_batch3d_step_sampled": (_st, [_vp, ctypes.c_uint64, ctypes.c_uint32, _dp]),
    "orr_batch3d_forces": (_st, [_vp, _dp]),
    "orr_batch3d_tune": (_st, [_vp, ctypes.c_uint32, ctypes.POINTER(abi.CBatchSchedule), ctypes.c_uint32, _u32p]),
    "orr_batch3d_synchronize": (_st, [_vp]),
    "orr_batch3d_stream": (_st, [_vp, ctypes.POINTER(_vp)]),
    "orr_batch3d_launch_count": (_st, [_vp, _u64p]),
    "orr_serve_create": (_st, [ctypes.POINTER(abi.CServeOptions), ctypes.POINTER(_vp)]),
    "orr_serve_destroy": (None, [_vp]),
    "orr_serve_last_error": (ctypes.c_char_p, [_vp]),
    "orr_serve_submit": (_st, [_vp, ctypes.POINTER(abi.CSolveRequest), _u64p]),
    "orr_serve_poll": (_st, [_vp, ctypes.c_uint64, ctypes.POINTER(abi.CSolveResult)]),
    "orr_serve_wait": (_st, [_vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(abi.CSolveResult)]),
    "orr_serve_drain": (_st, [_vp, ctypes.c_double]),
    "orr_serve_stats": (_st, [_vp, ctypes.POINTER(abi.CServeStatistics)]),
    "orr_grid_around": (_st, [_dp, _dp, ctypes.c_double, ctypes.c_uint64, ctypes.POINTER(abi.CGridSpec)]),
    "orr_voxelize": (_st, [ctypes.POINTER(abi.CMesh), ctypes.POINTER(abi.CGridSpec), ctypes.c_double, ctypes.c_int32,
                           _u8p, _dp, _dp]),
    "orr_signed_distance_band": (_st, [ctypes.POINTER(abi.CMesh), ctypes.POINTER(abi.CGridSpec), _u8p,
                                       ctypes.c_uint64, ctypes.c_double, ctypes.c_int32, _dp, _u8p, _dp, _dp]),
}


def library_path() -> str:
    from . import build
    return build.LIBRARY


def lib():
    """The loaded native library (built on first use when absent)."""
    global _LIB
    with _LOCK:
        if _LIB is None:
            path = library_path()
            if not os.path.exists(path):
                from . import build
                build.build()
            handle = ctypes.CDLL(path)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _LIB = handle
        return _LIB


class LbmError(RuntimeError):
    """A refused or failed call: ``status`` is the orr_status, the message the library's text."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int, message_fn) -> None:
    if status != abi.ORR_OK:
        msg = message_fn()
        if isinstance(msg, bytes):
            msg = msg.decode(errors="replace")
        raise LbmError(status, msg)


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)
