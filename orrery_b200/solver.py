"""Device lattice solvers, shaped like the reference's solver seam.

``make_gpu_solver(config, mask)`` returns a solver with the members of the
reference's ``Lbm3DSolver`` (src/aero/lbm3d/include/orrery/aero/lbm3d/lbm3d.h:196-232)
and ``Lbm2DSolver`` (src/aero/lbm/include/orrery/aero/lbm/lbm2d.h:173-202).  The
reference returns ``core::Result``; here a refusal raises ``LbmError`` with the
reference's message text.  Every call goes through the C ABI of
include/orrery_lbm.h.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import abi
from ._native import LbmError, check, lib, ptr
from .lbm3d import Lbm2DConfig, Lbm3DConfig
from .masks import SolidMask2D, SolidMask3D

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)

STORAGE_BYTES = {"f32": 4, "f16": 2, "bf16": 2, "f64": 8}


@dataclass
class MacroFields3D:
    """MacroFields3D (lbm3d.h:130-139)."""
    nx: int
    ny: int
    nz: int
    density: np.ndarray
    velocity_x: np.ndarray
    velocity_y: np.ndarray
    velocity_z: np.ndarray
    solid: np.ndarray


@dataclass
class MacroFields2D:
    """MacroFields2D (lbm2d.h:108-115)."""
    nx: int
    ny: int
    density: np.ndarray
    velocity_x: np.ndarray
    velocity_y: np.ndarray
    solid: np.ndarray


@dataclass
class Force3D:
    """Force3D (lbm3d.h:147-150): force and moment about the lattice origin."""
    force: np.ndarray
    moment: np.ndarray


@dataclass
class Force2D:
    """Force2D (lbm2d.h:128-132)."""
    x: float
    y: float
    moment: float


def _options(storage: str, allow_high_mach: bool, device: int, block_x: int, kernel: str = "auto",
             stages: int = 0, nodes_per_thread: int = 0) -> abi.CSolverOptions:
    if storage not in abi.STORAGE_NAMES:
        raise ValueError(f"unknown storage {storage!r}; one of {sorted(abi.STORAGE_NAMES)}")
    if kernel not in abi.KERNEL_NAMES:
        raise ValueError(f"unknown step kernel {kernel!r}; one of {sorted(abi.KERNEL_NAMES)}")
    o = abi.CSolverOptions()
    o.storage = abi.STORAGE_NAMES[storage]
    o.allow_high_mach = 1 if allow_high_mach else 0
    o.device = int(device)
    o.block_x = int(block_x)
    o.kernel = abi.KERNEL_NAMES[kernel]
    o.stages = int(stages)
    o.nodes_per_thread = int(nodes_per_thread)
    return o


def validate(config, mask, storage: str = "f32", allow_high_mach: bool = False) -> str | None:
    """validate() plus the device checks: the refusal text, or None when accepted."""
    L = lib()
    opts = _options(storage, allow_high_mach, 0, 0)
    msg = ctypes.create_string_buffer(1024)
    c = config.to_c()
    solid = np.ascontiguousarray(mask.solid, dtype=np.uint8)
    if isinstance(config, Lbm3DConfig):
        if solid.size != config.cells:
            return "lbm3d: the solid mask does not match the lattice size"
        dist = None if getattr(mask, "distance", None) is None else np.ascontiguousarray(mask.distance, np.float64)
        st = L.orr_lbm3d_validate(ctypes.byref(c), ptr(solid, _u8p), ptr(dist, _dp), ctypes.byref(opts), msg, 1024)
    else:
        if solid.size != config.cells:
            return "lbm2d: the solid mask does not match the lattice size"
        st = L.orr_lbm2d_validate(ctypes.byref(c), ptr(solid, _u8p), ctypes.byref(opts), msg, 1024)
    return None if st == abi.ORR_OK else msg.value.decode()


def memory_bytes(config: Lbm3DConfig, links: int, boundary_nodes: int, storage: str = "f32") -> int:
    out = ctypes.c_uint64()
    L = lib()
    c = config.to_c()
    check(L.orr_lbm3d_memory_bytes(ctypes.byref(c), links, boundary_nodes, abi.STORAGE_NAMES[storage],
                                   ctypes.byref(out)), L.orr_last_error)
    return out.value


def plan3d(config: Lbm3DConfig, mask: SolidMask3D):
    """Host-only planning (no device): boundary links with their wall fractions
    and node counts.  Returns (cell, direction, q, fluid, boundary_nodes)."""
    L = lib()
    c = config.to_c()
    solid = np.ascontiguousarray(mask.solid, dtype=np.uint8).reshape(-1)
    dist = None if mask.distance is None else np.ascontiguousarray(mask.distance, np.float64).reshape(-1)
    n, fluid, bnodes = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    check(L.orr_lbm3d_plan(ctypes.byref(c), ptr(solid, _u8p), ptr(dist, _dp), ctypes.byref(n), ctypes.byref(fluid),
                           ctypes.byref(bnodes), None, None, None), L.orr_last_error)
    cell = np.empty(n.value, np.uint32)
    d = np.empty(n.value, np.uint32)
    q = np.empty(n.value)
    check(L.orr_lbm3d_plan(ctypes.byref(c), ptr(solid, _u8p), ptr(dist, _dp), None, None, None,
                           ptr(cell, _u32p), ptr(d, _u32p), ptr(q, _dp)), L.orr_last_error)
    return cell, d, q, fluid.value, bnodes.value


class CudaLbm3D:
    """A D3Q19 device solver (the reference's GpuLbm3D behind Lbm3DSolver)."""

    q = 19

    def __init__(self, config: Lbm3DConfig, mask: SolidMask3D, storage: str = "f32",
                 allow_high_mach: bool = False, device: int = 0, block_x: int = 0,
                 kernel: str = "auto", stages: int = 0, nodes_per_thread: int = 0):
        self._lib = lib()
        self._h = None
        self.config = config
        self.mask = mask
        self.storage = storage
        self.cells = config.cells
        solid = np.ascontiguousarray(mask.solid, dtype=np.uint8).reshape(-1)
        if solid.size != self.cells:
            raise LbmError(abi.ORR_ERR_INVALID, "lbm3d: the solid mask does not match the lattice size")
        dist = None if mask.distance is None else np.ascontiguousarray(mask.distance, np.float64).reshape(-1)
        self._solid = solid
        opts = _options(storage, allow_high_mach, device, block_x, kernel, stages, nodes_per_thread)
        c = config.to_c()
        h = ctypes.c_void_p()
        check(self._lib.orr_lbm3d_create(ctypes.byref(c), ptr(solid, _u8p), ptr(dist, _dp), ctypes.byref(opts),
                                         ctypes.byref(h)), self._lib.orr_last_error)
        self._h = h

    def close(self) -> None:
        if self._h is not None:
            self._lib.orr_lbm3d_destroy(self._h)
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

    def _check(self, status: int) -> None:
        check(status, lambda: self._lib.orr_lbm3d_last_error(self._h))

    # -- Lbm3DSolver members --------------------------------------------
    def steps(self) -> int:
        out = ctypes.c_uint64()
        self._check(self._lib.orr_lbm3d_steps(self._h, ctypes.byref(out)))
        return out.value

    def initialize(self, rho=None, ux=None, uy=None, uz=None) -> None:
        """Equilibrium of the given fields (arrays of nx*ny*nz, or a callable
        ``state(x, y, z) -> (rho, ux, uy, uz)`` vectorised over node arrays);
        no arguments restore the uniform inlet state."""
        if callable(rho):
            nx, ny, nz = self.config.nx, self.config.ny, self.config.nz
            z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
            vals = rho(x.reshape(-1), y.reshape(-1), z.reshape(-1))
            rho, ux, uy, uz = (np.broadcast_to(np.asarray(v, np.float64), (self.cells,)) for v in vals)
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64).reshape(-1) for a in (rho, ux, uy, uz)]
        self._check(self._lib.orr_lbm3d_initialize(self._h, *[ptr(a, _dp) for a in arrs]))

    def step(self, count: int = 1) -> None:
        self._check(self._lib.orr_lbm3d_step(self._h, int(count)))

    def set_inlet_velocity(self, velocity) -> None:
        v = np.ascontiguousarray(velocity, np.float64)
        self._check(self._lib.orr_lbm3d_set_inlet_velocity(self._h, ptr(v, _dp)))

    def inlet_velocity(self) -> np.ndarray:
        v = np.empty(3)
        self._check(self._lib.orr_lbm3d_inlet_velocity(self._h, ptr(v, _dp)))
        return v

    def macroscopic(self, out: MacroFields3D | None = None) -> MacroFields3D:
        """Density and velocity of every node.  With `out` (the fields of an
        earlier call on a lattice of this size) the values are written into
        its arrays, which saves the page faults of fresh ones when fields
        are read back repeatedly."""
        if out is None:
            planes = [np.empty(self.cells) for _ in range(4)]
        else:
            planes = [out.density, out.velocity_x, out.velocity_y, out.velocity_z]
            if any(a.dtype != np.float64 or a.size != self.cells or not a.flags.c_contiguous or not a.flags.writeable
                   for a in planes):
                raise LbmError(abi.ORR_ERR_INVALID, "lbm3d: macroscopic(out) needs four writable contiguous "
                                                    "float64 arrays of nx*ny*nz values")
        self._check(self._lib.orr_lbm3d_macroscopic(self._h, *[ptr(a, _dp) for a in planes]))
        if out is not None:
            # the shape and mask of this solver, whichever solver of as many
            # nodes filled `out` before
            out.nx, out.ny, out.nz = self.config.nx, self.config.ny, self.config.nz
            if isinstance(out.solid, np.ndarray) and out.solid.shape == self._solid.shape \
                    and out.solid.dtype == self._solid.dtype and out.solid.flags.writeable:
                np.copyto(out.solid, self._solid)
            else:
                out.solid = self._solid.copy()
            return out
        return MacroFields3D(self.config.nx, self.config.ny, self.config.nz, *planes, self._solid.copy())

    def populations(self, out: np.ndarray | None = None) -> np.ndarray:
        """The 19 populations of every node (unshifted), direction-major; into
        `out` (a writable contiguous float64 array of 19*nx*ny*nz values)
        when given."""
        if out is None:
            f = np.empty(self.q * self.cells)
        else:
            f = out
            if f.dtype != np.float64 or f.size != self.q * self.cells or not f.flags.c_contiguous or \
                    not f.flags.writeable:
                raise LbmError(abi.ORR_ERR_INVALID, "lbm3d: populations(out) needs a writable contiguous "
                                                    "float64 array of 19*nx*ny*nz values")
        self._check(self._lib.orr_lbm3d_populations(self._h, ptr(f, _dp)))
        return f

    def force(self) -> Force3D:
        out = np.empty(6)
        self._check(self._lib.orr_lbm3d_force(self._h, ptr(out, _dp)))
        return Force3D(out[:3].copy(), out[3:].copy())

    def mass(self) -> float:
        out = ctypes.c_double()
        self._check(self._lib.orr_lbm3d_mass(self._h, ctypes.byref(out)))
        return out.value

    def links(self):
        n = ctypes.c_uint64()
        self._check(self._lib.orr_lbm3d_link_count(self._h, ctypes.byref(n)))
        cell = np.empty(n.value, np.uint32)
        d = np.empty(n.value, np.uint32)
        q = np.empty(n.value)
        self._check(self._lib.orr_lbm3d_links(self._h, ptr(cell, _u32p), ptr(d, _u32p), ptr(q, _dp)))
        return cell, d, q

    # -- device-side extras ---------------------------------------------
    def node_counts(self):
        fluid, boundary = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._lib.orr_lbm3d_node_counts(self._h, ctypes.byref(fluid), ctypes.byref(boundary)))
        return fluid.value, boundary.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.orr_lbm3d_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        n = ctypes.c_uint64()
        self._check(self._lib.orr_lbm3d_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def request_stall(self, cta: int = 0) -> None:
        """Test hook of the staged step's bounded waits: the next staged
        launch's CTA `cta` withholds its first span's copies, so the next
        read-back raises the timeout error until initialize()."""
        self._check(self._lib.orr_lbm3d_request_stall(self._h, int(cta)))

    def kernel_info(self) -> dict:
        """The step kernel this solver runs and its launch shape."""
        k = abi.CKernelInfo()
        self._check(self._lib.orr_lbm3d_kernel_info(self._h, ctypes.byref(k)))
        names = {v: n for n, v in abi.KERNEL_NAMES.items()}
        return {"kernel": names.get(k.kernel, str(k.kernel)), "block": k.block, "stages": k.stages,
                "grid": k.grid, "ctas_per_sm": k.ctas_per_sm, "registers": k.registers,
                "shared_bytes": k.shared_bytes, "nodes_per_thread": k.nodes_per_thread,
                "staged_items": k.staged_items,
                "direct_items": k.direct_items}


class CudaLbm2D:
    """A D2Q9 device solver (the reference's GpuLbm2D behind Lbm2DSolver)."""

    q = 9

    def __init__(self, config: Lbm2DConfig, mask: SolidMask2D, storage: str = "f32",
                 allow_high_mach: bool = False, device: int = 0, block_x: int = 0):
        self._lib = lib()
        self._h = None
        self.config = config
        self.mask = mask
        self.storage = storage
        self.cells = config.cells
        solid = np.ascontiguousarray(mask.solid, dtype=np.uint8).reshape(-1)
        if solid.size != self.cells:
            raise LbmError(abi.ORR_ERR_INVALID, "lbm2d: the solid mask does not match the lattice size")
        self._solid = solid
        opts = _options(storage, allow_high_mach, device, block_x)
        c = config.to_c()
        h = ctypes.c_void_p()
        check(self._lib.orr_lbm2d_create(ctypes.byref(c), ptr(solid, _u8p), ctypes.byref(opts), ctypes.byref(h)),
              self._lib.orr_last_error)
        self._h = h

    def close(self) -> None:
        if self._h is not None:
            self._lib.orr_lbm2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int) -> None:
        check(status, lambda: self._lib.orr_lbm2d_last_error(self._h))

    def steps(self) -> int:
        out = ctypes.c_uint64()
        self._check(self._lib.orr_lbm2d_steps(self._h, ctypes.byref(out)))
        return out.value

    def initialize(self, rho=None, ux=None, uy=None) -> None:
        if callable(rho):
            nx, ny = self.config.nx, self.config.ny
            y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
            vals = rho(x.reshape(-1), y.reshape(-1))
            rho, ux, uy = (np.broadcast_to(np.asarray(v, np.float64), (self.cells,)) for v in vals)
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64).reshape(-1) for a in (rho, ux, uy)]
        self._check(self._lib.orr_lbm2d_initialize(self._h, *[ptr(a, _dp) for a in arrs]))

    def step(self, count: int = 1) -> None:
        self._check(self._lib.orr_lbm2d_step(self._h, int(count)))

    def macroscopic(self) -> MacroFields2D:
        out = [np.empty(self.cells) for _ in range(3)]
        self._check(self._lib.orr_lbm2d_macroscopic(self._h, *[ptr(a, _dp) for a in out]))
        return MacroFields2D(self.config.nx, self.config.ny, *out, self._solid.copy())

    def populations(self) -> np.ndarray:
        f = np.empty(self.q * self.cells)
        self._check(self._lib.orr_lbm2d_populations(self._h, ptr(f, _dp)))
        return f

    def force(self) -> Force2D:
        out = np.empty(3)
        self._check(self._lib.orr_lbm2d_force(self._h, ptr(out, _dp)))
        return Force2D(float(out[0]), float(out[1]), float(out[2]))

    def mass(self) -> float:
        out = ctypes.c_double()
        self._check(self._lib.orr_lbm2d_mass(self._h, ctypes.byref(out)))
        return out.value

    def links(self):
        n = ctypes.c_uint64()
        self._check(self._lib.orr_lbm2d_link_count(self._h, ctypes.byref(n)))
        cell = np.empty(n.value, np.uint32)
        d = np.empty(n.value, np.uint32)
        self._check(self._lib.orr_lbm2d_links(self._h, ptr(cell, _u32p), ptr(d, _u32p)))
        return cell, d

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.orr_lbm2d_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        n = ctypes.c_uint64()
        self._check(self._lib.orr_lbm2d_launch_count(self._h, ctypes.byref(n)))
        return n.value


def make_gpu_solver(config, mask, storage: str = "f32", allow_high_mach: bool = False,
                    device: int = 0, block_x: int = 0, kernel: str = "auto", stages: int = 0,
                    nodes_per_thread: int = 0):
    """make_gpu_solver (lbm3d.h:246-247; lbm2d.h:211-212) on the CUDA path.
    `kernel` and `stages` choose the D3Q19 step kernel (ignored in 2D)."""
    if isinstance(config, Lbm3DConfig):
        return CudaLbm3D(config, mask, storage, allow_high_mach, device, block_x, kernel, stages,
                         nodes_per_thread)
    if isinstance(config, Lbm2DConfig):
        return CudaLbm2D(config, mask, storage, allow_high_mach, device, block_x)
    raise TypeError("config must be an Lbm3DConfig or an Lbm2DConfig")
