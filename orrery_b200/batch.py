"""Batches of D3Q19 solvers advanced together (orr_batch3d_* of the C ABI).

A batch holds ordinary ``CudaLbm3D`` solvers and steps all of them with one
persistent launch per step (or a captured graph of per-lattice launches),
chosen by the autotuner ``tune()``.  Each member's populations are exactly
those its own steps would give; forces are summed in a fixed order, so a
member's force is the same alone and in any mix.  While a solver belongs to
a batch its own ``step()`` is refused.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from ._native import check, lib, ptr
from .solver import CudaLbm3D

_dp = ctypes.POINTER(ctypes.c_double)
_KERNELS = {v: n for n, v in abi.KERNEL_NAMES.items()}


def _schedule_dict(s: abi.CBatchSchedule) -> dict:
    return {"kernel": _KERNELS.get(s.kernel, str(s.kernel)), "block": s.block, "stages": s.stages,
            "nodes_per_thread": s.nodes_per_thread, "branches": s.branches, "grid": s.grid,
            "ms_per_step": s.ms_per_step}


class CudaBatch3D:
    def __init__(self, device: int = 0):
        self._lib = lib()
        self._h = None
        self.members: list[CudaLbm3D] = []
        h = ctypes.c_void_p()
        check(self._lib.orr_batch3d_create(int(device), ctypes.byref(h)), self._lib.orr_last_error)
        self._h = h

    def _check(self, status: int) -> None:
        check(status, lambda: self._lib.orr_batch3d_last_error(self._h))

    def close(self) -> None:
        if self._h is not None:
            self._lib.orr_batch3d_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, solver: CudaLbm3D) -> None:
        self._check(self._lib.orr_batch3d_add(self._h, solver._h))
        self.members.append(solver)

    def remove(self, solver: CudaLbm3D) -> None:
        self._check(self._lib.orr_batch3d_remove(self._h, solver._h))
        self.members.remove(solver)

    def size(self) -> tuple[int, int]:
        n, cells = ctypes.c_uint32(), ctypes.c_uint64()
        self._check(self._lib.orr_batch3d_size(self._h, ctypes.byref(n), ctypes.byref(cells)))
        return n.value, cells.value

    def set_schedule(self, kernel: str = "staged", block: int = 256, stages: int = 0,
                     nodes_per_thread: int = 0, branches: int = 0) -> None:
        s = abi.CBatchSchedule()
        s.kernel = abi.KERNEL_NAMES[kernel]
        s.block = int(block)
        s.stages = int(stages)
        s.nodes_per_thread = int(nodes_per_thread)
        s.branches = int(branches)
        self._check(self._lib.orr_batch3d_set_schedule(self._h, ctypes.byref(s)))

    def schedule(self) -> dict:
        s = abi.CBatchSchedule()
        self._check(self._lib.orr_batch3d_schedule(self._h, ctypes.byref(s)))
        return _schedule_dict(s)

    def step(self, count: int = 1) -> None:
        self._check(self._lib.orr_batch3d_step(self._h, int(count)))

    def step_sampled(self, count: int, sample_every: int = 10) -> np.ndarray:
        """Steps with the force sampled every `sample_every` steps; returns the
        (members, 6) sums of force and moment over the samples."""
        out = np.zeros((len(self.members), 6))
        self._check(self._lib.orr_batch3d_step_sampled(self._h, int(count), int(sample_every),
                                                       ptr(out, _dp)))
        return out

    def forces(self) -> np.ndarray:
        """(members, 6) force and moment about the lattice origin, fixed-order sums."""
        out = np.zeros((len(self.members), 6))
        self._check(self._lib.orr_batch3d_forces(self._h, ptr(out, _dp)))
        return out

    def tune(self, graphs_per_trial: int = 2) -> list[dict]:
        """Times every candidate schedule on the batch (real steps) and keeps the fastest."""
        trials = (abi.CBatchSchedule * 16)()
        n = ctypes.c_uint32()
        self._check(self._lib.orr_batch3d_tune(self._h, int(graphs_per_trial), trials, 16, ctypes.byref(n)))
        return [_schedule_dict(trials[k]) for k in range(n.value)]

    def synchronize(self) -> None:
        self._check(self._lib.orr_batch3d_synchronize(self._h))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.orr_batch3d_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        n = ctypes.c_uint64()
        self._check(self._lib.orr_batch3d_launch_count(self._h, ctypes.byref(n)))
        return n.value
