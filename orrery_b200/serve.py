"""Serving of D3Q19 drag solves with continuous batching (orr_serve_* of the C ABI).

``Server.submit(workload, ...)`` queues a solve and returns its id at once;
a worker thread in the library admits queued solves against the device-memory
budget and slot count, runs every admitted lattice in one batch, and retires
each solve when the mean Cd of its last window differs from the previous
window's by less than the tolerance (or at its step cap).  ``poll``/``wait``
return a solve's result, ``stats()`` the latency percentiles and throughput.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from ._native import LbmError, check, lib, ptr
from .workloads import Workload3D

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _result(r: abi.CSolveResult) -> dict:
    return {"state": abi.SOLVE_STATES.get(r.state, str(r.state)), "steps": r.steps, "cd": r.cd, "cl": r.cl,
            "cm": r.cm, "delta_cd": r.delta_cd, "force": list(r.force), "moment": list(r.moment),
            "arrival_s": r.arrival_s, "admitted_s": r.admitted_s, "finished_s": r.finished_s,
            "latency_s": r.finished_s - r.arrival_s if r.finished_s > 0 else None,
            "device_bytes": r.device_bytes, "message": r.message.decode(errors="replace")}


# The reference adapter's steady criterion: every force range over the
# window within 1e-3 of the mean drag (kSteadyResidual,
# src/aero/lbm3d/lbm_aero_solver3d.cpp:25, forces_settled_3d at :61-80).
STEADY_RANGE = 1e-3


class Server:
    def __init__(self, storage: str = "f32", device: int = 0, memory_budget: float = 150e9,
                 max_active: int = 64, chunk_steps: int = 100, sample_every: int = 10,
                 kernel: str = "auto", block: int = 0, stages: int = 0, branches: int = 0):
        self._lib = lib()
        self._h = None
        o = abi.CServeOptions()
        o.storage = abi.STORAGE_NAMES[storage]
        o.device = int(device)
        o.memory_budget = int(memory_budget)
        o.max_active = int(max_active)
        o.chunk_steps = int(chunk_steps)
        o.sample_every = int(sample_every)
        o.kernel = abi.KERNEL_NAMES[kernel]
        o.block = int(block)
        o.stages = int(stages)
        o.branches = int(branches)
        h = ctypes.c_void_p()
        check(self._lib.orr_serve_create(ctypes.byref(o), ctypes.byref(h)), self._lib.orr_last_error)
        self._h = h
        self.storage = storage

    def _check(self, status: int) -> None:
        check(status, lambda: self._lib.orr_serve_last_error(self._h))

    def close(self) -> None:
        if self._h is not None:
            self._lib.orr_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, w: Workload3D, window: int = 500, tolerance: float = 1e-4, max_steps: int = 0,
               initial_state: bool = True, moment_centre=(0.0, 0.0, 0.0), fixed_steps: bool = False,
               ramp_steps: float = 0.0, steady_range: float = 0.0) -> int:
        """Queues the solve of workload `w`; returns its id.  Without
        `initial_state` the solve starts from the uniform inlet state.
        `fixed_steps`: run exactly `max_steps` steps and report the means over
        the last `window` steps.  `ramp_steps` > 0: start at rest with the
        reference adapter's gradual start of the inlet velocity.
        `steady_range` > 0: a window settles only when its force ranges are
        within this fraction of the mean drag force as well (the reference
        adapter's steady test; STEADY_RANGE is its bound); 0, the default,
        leaves the |delta Cd| rule alone."""
        c = w.config.to_c()
        solid = np.ascontiguousarray(w.mask.solid, np.uint8).reshape(-1)
        dist = None if w.mask.distance is None else np.ascontiguousarray(w.mask.distance, np.float64).reshape(-1)
        fields = [np.ascontiguousarray(a, np.float64).reshape(-1) for a in (w.rho, w.ux, w.uy, w.uz)] \
            if initial_state and w.rho is not None and not ramp_steps > 0 else [None] * 4
        r = abi.CSolveRequest()
        r.config = ctypes.pointer(c)
        r.solid = ptr(solid, _u8p)
        r.distance = ptr(dist, _dp)
        r.rho, r.ux, r.uy, r.uz = (ptr(a, _dp) for a in fields)
        r.allow_high_mach = 1 if w.allow_high_mach else 0
        r.sample_every = 0
        r.window = int(window)
        r.tolerance = float(tolerance)
        r.max_steps = int(max_steps)
        r.reference_area = float(w.reference_area)
        r.reference_length = float(w.reference_length)
        r.moment_centre = (ctypes.c_double * 3)(*[float(v) for v in moment_centre])
        r.mode = abi.ORR_RUN_FIXED_STEPS if fixed_steps else abi.ORR_RUN_UNTIL_SETTLED
        r.ramp_steps = float(ramp_steps)
        r.steady_range = float(steady_range)
        out = ctypes.c_uint64()
        self._check(self._lib.orr_serve_submit(self._h, ctypes.byref(r), ctypes.byref(out)))
        return out.value

    def poll(self, rid: int) -> dict:
        r = abi.CSolveResult()
        self._check(self._lib.orr_serve_poll(self._h, int(rid), ctypes.byref(r)))
        return _result(r)

    def wait(self, rid: int, timeout: float = 600.0) -> dict:
        r = abi.CSolveResult()
        self._check(self._lib.orr_serve_wait(self._h, int(rid), float(timeout), ctypes.byref(r)))
        return _result(r)

    def drain(self, timeout: float = 3600.0) -> None:
        self._check(self._lib.orr_serve_drain(self._h, float(timeout)))

    def stats(self) -> dict:
        t = abi.CServeStatistics()
        self._check(self._lib.orr_serve_stats(self._h, ctypes.byref(t)))
        return {k: (getattr(t, k).decode(errors="replace") if k == "message" else getattr(t, k))
                for k, _ in t._fields_}


__all__ = ["Server", "LbmError"]
