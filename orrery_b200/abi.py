"""ctypes mirror of include/orrery_lbm.h: the C structs and enums of the ABI.

Plain data definitions only; loading the native library lives in
``orrery_b200._native``.
"""
from __future__ import annotations

import ctypes

# Status codes.
ORR_OK = 0
ORR_ERR_INVALID = 1
ORR_ERR_MEMORY = 2
ORR_ERR_CUDA = 3
ORR_ERR_STATE = 4
ORR_ERR_TIMEOUT = 5
ORR_ERR_DIVERGED = 6
ORR_ERR_NO_DEVICE = 7

# Wall kinds, x boundary, outlet, solid wall, storage.
ORR_WALL_PERIODIC, ORR_WALL_SLIP, ORR_WALL_NO_SLIP = 0, 1, 2
ORR_X_PERIODIC, ORR_X_INFLOW_OUTFLOW = 0, 1
ORR_OUTLET_CONVECTIVE, ORR_OUTLET_EXTRAPOLATION = 0, 1
ORR_SOLID_HALFWAY, ORR_SOLID_INTERPOLATED = 0, 1
ORR_STORAGE_F32, ORR_STORAGE_F16, ORR_STORAGE_BF16, ORR_STORAGE_F64 = 0, 1, 2, 3

STORAGE_NAMES = {"f32": ORR_STORAGE_F32, "f16": ORR_STORAGE_F16, "bf16": ORR_STORAGE_BF16,
                 "f64": ORR_STORAGE_F64}


class CWall(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("pad_", ctypes.c_int32), ("velocity_x", ctypes.c_double)]


class CLbm3DConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_uint64), ("ny", ctypes.c_uint64), ("nz", ctypes.c_uint64),
        ("tau", ctypes.c_double),
        ("x_boundary", ctypes.c_int32), ("outlet", ctypes.c_int32),
        ("y_low", CWall), ("y_high", CWall), ("z_low", CWall), ("z_high", CWall),
        ("inlet_ux", ctypes.c_double), ("inlet_uy", ctypes.c_double), ("inlet_uz", ctypes.c_double),
        ("body_force_x", ctypes.c_double), ("body_force_y", ctypes.c_double),
        ("body_force_z", ctypes.c_double),
        ("smagorinsky_enabled", ctypes.c_int32), ("solid_wall", ctypes.c_int32),
        ("smagorinsky_constant", ctypes.c_double),
        ("sponge_strength", ctypes.c_double),
        ("sponge_inlet", ctypes.c_uint64), ("sponge_outlet", ctypes.c_uint64),
        ("sponge_sides", ctypes.c_uint64),
    ]


class CLbm2DConfig(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_uint64), ("ny", ctypes.c_uint64),
        ("tau", ctypes.c_double),
        ("x_boundary", ctypes.c_int32), ("outlet", ctypes.c_int32),
        ("bottom", CWall), ("top", CWall),
        ("inlet_ux", ctypes.c_double), ("inlet_uy", ctypes.c_double),
        ("body_force_x", ctypes.c_double), ("body_force_y", ctypes.c_double),
        ("smagorinsky_enabled", ctypes.c_int32), ("pad_", ctypes.c_int32),
        ("smagorinsky_constant", ctypes.c_double),
    ]


class CForceLinks(ctypes.Structure):
    """orr_force_links: device inputs of orr_lbm3d_force_static."""
    _fields_ = [("nx", ctypes.c_uint64), ("ny", ctypes.c_uint64), ("nz", ctypes.c_uint64),
                ("storage", ctypes.c_int32), ("device", ctypes.c_int32),
                ("populations", ctypes.c_void_p), ("link_cell", ctypes.c_void_p),
                ("link_dir", ctypes.c_void_p), ("link_q", ctypes.c_void_p),
                ("links", ctypes.c_uint64), ("stream", ctypes.c_void_p)]


ORR_FORCE_STATIC_MAX_LINKS = 8388608


ORR_KERNEL_AUTO, ORR_KERNEL_ROWS, ORR_KERNEL_STAGED, ORR_KERNEL_TILED = 0, 1, 2, 3
KERNEL_NAMES = {"auto": ORR_KERNEL_AUTO, "rows": ORR_KERNEL_ROWS, "staged": ORR_KERNEL_STAGED,
                "tiled": ORR_KERNEL_TILED}


class CKernelInfo(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("block", ctypes.c_uint32), ("stages", ctypes.c_uint32),
                ("grid", ctypes.c_uint32), ("ctas_per_sm", ctypes.c_int32), ("registers", ctypes.c_int32),
                ("shared_bytes", ctypes.c_uint32), ("nodes_per_thread", ctypes.c_uint32),
                ("staged_items", ctypes.c_uint64), ("direct_items", ctypes.c_uint64)]


class CSolverOptions(ctypes.Structure):
    _fields_ = [("storage", ctypes.c_int32), ("allow_high_mach", ctypes.c_int32),
                ("device", ctypes.c_int32), ("block_x", ctypes.c_int32),
                ("kernel", ctypes.c_int32), ("stages", ctypes.c_int32),
                ("nodes_per_thread", ctypes.c_int32)]


class CBatchSchedule(ctypes.Structure):
    """orr_batch_schedule."""
    _fields_ = [("kernel", ctypes.c_int32), ("block", ctypes.c_uint32), ("stages", ctypes.c_uint32),
                ("grid", ctypes.c_uint32), ("nodes_per_thread", ctypes.c_uint32), ("branches", ctypes.c_uint32),
                ("ms_per_step", ctypes.c_double)]


class CServeOptions(ctypes.Structure):
    """orr_serve_options."""
    _fields_ = [("storage", ctypes.c_int32), ("device", ctypes.c_int32), ("memory_budget", ctypes.c_uint64),
                ("max_active", ctypes.c_uint32), ("chunk_steps", ctypes.c_uint32),
                ("sample_every", ctypes.c_uint32), ("kernel", ctypes.c_int32), ("block", ctypes.c_uint32),
                ("stages", ctypes.c_uint32), ("branches", ctypes.c_uint32)]


class CSolveRequest(ctypes.Structure):
    """orr_solve_request."""
    _fields_ = [("config", ctypes.POINTER(CLbm3DConfig)), ("solid", ctypes.POINTER(ctypes.c_uint8)),
                ("distance", ctypes.POINTER(ctypes.c_double)), ("rho", ctypes.POINTER(ctypes.c_double)),
                ("ux", ctypes.POINTER(ctypes.c_double)), ("uy", ctypes.POINTER(ctypes.c_double)),
                ("uz", ctypes.POINTER(ctypes.c_double)), ("allow_high_mach", ctypes.c_int32),
                ("sample_every", ctypes.c_uint32), ("window", ctypes.c_uint32), ("mode", ctypes.c_uint32),
                ("tolerance", ctypes.c_double), ("max_steps", ctypes.c_uint64),
                ("reference_area", ctypes.c_double), ("reference_length", ctypes.c_double),
                ("moment_centre", ctypes.c_double * 3), ("ramp_steps", ctypes.c_double),
                ("steady_range", ctypes.c_double)]


ORR_RUN_UNTIL_SETTLED, ORR_RUN_FIXED_STEPS = 0, 1
ORR_SOLVE_QUEUED, ORR_SOLVE_RUNNING, ORR_SOLVE_CONVERGED, ORR_SOLVE_CAPPED, ORR_SOLVE_FAILED = 0, 1, 2, 3, 4
ORR_SOLVE_COMPLETED = 5
SOLVE_STATES = {0: "queued", 1: "running", 2: "converged", 3: "capped", 4: "failed", 5: "completed"}


class CSolveResult(ctypes.Structure):
    """orr_solve_result."""
    _fields_ = [("state", ctypes.c_int32), ("reserved", ctypes.c_int32), ("steps", ctypes.c_uint64),
                ("cd", ctypes.c_double), ("cl", ctypes.c_double), ("cm", ctypes.c_double),
                ("delta_cd", ctypes.c_double), ("force", ctypes.c_double * 3), ("moment", ctypes.c_double * 3),
                ("arrival_s", ctypes.c_double), ("admitted_s", ctypes.c_double), ("finished_s", ctypes.c_double),
                ("device_bytes", ctypes.c_uint64), ("message", ctypes.c_char * 160)]


class CServeStatistics(ctypes.Structure):
    """orr_serve_statistics."""
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("queued", ctypes.c_uint64), ("active", ctypes.c_uint64), ("latency_p50_s", ctypes.c_double),
                ("latency_p99_s", ctypes.c_double), ("latency_mean_s", ctypes.c_double),
                ("solves_per_second", ctypes.c_double), ("lattice_updates", ctypes.c_double),
                ("busy_seconds", ctypes.c_double), ("peak_device_bytes", ctypes.c_uint64),
                ("mean_active", ctypes.c_double), ("chunks", ctypes.c_uint64), ("worker_failed", ctypes.c_int32),
                ("message", ctypes.c_char * 160)]


class CGridSpec(ctypes.Structure):
    """orr_grid_spec (geom::GridSpec)."""
    _fields_ = [("origin", ctypes.c_double * 3), ("spacing", ctypes.c_double), ("nx", ctypes.c_uint64),
                ("ny", ctypes.c_uint64), ("nz", ctypes.c_uint64)]


class CMesh(ctypes.Structure):
    """orr_mesh (geom::TriangleMesh as flat arrays)."""
    _fields_ = [("vertices", ctypes.POINTER(ctypes.c_double)), ("vertex_count", ctypes.c_uint64),
                ("triangles", ctypes.POINTER(ctypes.c_uint32)), ("triangle_count", ctypes.c_uint64)]
