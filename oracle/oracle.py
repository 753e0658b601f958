"""Python access to the two CPU oracles of the LBM path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg, never by the product package.

``Restated3D`` / ``Restated2D``  the plain-C binary64 restatement
                                  (oracle/lbm_oracle.c, always buildable).
``Reference3D`` / ``Reference2D`` Orrery's own CpuLbm3D / CpuLbm2D compiled
                                  from the reference sources (oracle/_ref);
                                  present only where that build ran.
Both expose the same methods, shaped like the reference's Lbm3DSolver
(src/aero/lbm3d/include/orrery/aero/lbm3d/lbm3d.h:196-232).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from orrery_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED_SO = os.path.join(HERE, "_build", "liblbm_oracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libref_lbm.so")

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_vp = ctypes.c_void_p

_restated = None
_reference = None


def reference_tree(reference: str | None = None) -> str | None:
    """The reference source tree: `reference`, else $ORR_REFERENCE, else a
    checkout named ``reference`` beside this repository; None when none of
    them holds the LBM sources."""
    candidates = [reference, os.environ.get("ORR_REFERENCE"),
                  os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for ref in candidates:
        if ref and os.path.isdir(os.path.join(ref, "src", "aero", "lbm3d")):
            return os.path.abspath(ref)
    return None


def build(reference: str | None = None) -> None:
    """Builds the restatement, and the reference libraries when the reference
    tree is found (the adapter harness after the product library)."""
    env = dict(os.environ)
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True, env=env)
    ref = reference_tree(reference)
    if ref is not None:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True, env=env)
        subprocess.run(["make", "-s", "-C", HERE, "adapter", f"REF={ref}"], check=True, env=env)
        subprocess.run(["make", "-s", "-C", HERE, "backend", f"REF={ref}"], check=True, env=env)


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


def restated_lib():
    global _restated
    if _restated is None:
        if not os.path.exists(RESTATED_SO):
            build()
        lib = ctypes.CDLL(RESTATED_SO)
        lib.lo3_create.restype = _vp
        lib.lo3_create.argtypes = [ctypes.POINTER(abi.CLbm3DConfig), _u8p, _dp]
        lib.lo3_destroy.argtypes = [_vp]
        lib.lo3_initialize.argtypes = [_vp, _dp, _dp, _dp, _dp]
        lib.lo3_step.argtypes = [_vp, ctypes.c_uint64]
        lib.lo3_set_inlet.argtypes = [_vp, _dp]
        lib.lo3_populations.argtypes = [_vp, _dp]
        lib.lo3_force.argtypes = [_vp, _dp]
        lib.lo3_macroscopic.argtypes = [_vp, _dp, _dp, _dp, _dp]
        lib.lo3_mass.argtypes = [_vp]
        lib.lo3_mass.restype = ctypes.c_double
        lib.lo3_link_count.argtypes = [_vp]
        lib.lo3_link_count.restype = ctypes.c_uint64
        lib.lo3_links.argtypes = [_vp, _u32p, _u32p, _dp]
        lib.lo3_boundary_count.argtypes = [_vp]
        lib.lo3_boundary_count.restype = ctypes.c_uint64
        lib.lo2_create.restype = _vp
        lib.lo2_create.argtypes = [ctypes.POINTER(abi.CLbm2DConfig), _u8p]
        lib.lo2_destroy.argtypes = [_vp]
        lib.lo2_initialize.argtypes = [_vp, _dp, _dp, _dp]
        lib.lo2_step.argtypes = [_vp, ctypes.c_uint64]
        lib.lo2_populations.argtypes = [_vp, _dp]
        lib.lo2_force.argtypes = [_vp, _dp]
        lib.lo2_macroscopic.argtypes = [_vp, _dp, _dp, _dp]
        lib.lo2_mass.argtypes = [_vp]
        lib.lo2_mass.restype = ctypes.c_double
        lib.lo2_link_count.argtypes = [_vp]
        lib.lo2_link_count.restype = ctypes.c_uint64
        lib.lo2_links.argtypes = [_vp, _u32p, _u32p]
        lib.lo_set_threads.argtypes = [ctypes.c_int]
        lib.lo_threads.restype = ctypes.c_int
        _restated = lib
    return _restated


def reference_available() -> bool:
    return os.path.exists(REFERENCE_SO)


def reference_lib():
    global _reference
    if _reference is None:
        if not reference_available():
            raise FileNotFoundError(f"reference oracle not built: {REFERENCE_SO}")
        lib = ctypes.CDLL(REFERENCE_SO)
        c3 = ctypes.POINTER(abi.CLbm3DConfig)
        c2 = ctypes.POINTER(abi.CLbm2DConfig)
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_threads.restype = ctypes.c_int
        lib.ref3d_validate.argtypes = [c3, _u8p, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref3d_create.restype = _vp
        lib.ref3d_create.argtypes = [c3, _u8p, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref3d_destroy.argtypes = [_vp]
        lib.ref3d_initialize.argtypes = [_vp, _dp, _dp, _dp, _dp]
        lib.ref3d_step.argtypes = [_vp, ctypes.c_uint64]
        lib.ref3d_set_inlet.argtypes = [_vp, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref3d_populations.argtypes = [_vp, _dp]
        lib.ref3d_force.argtypes = [_vp, _dp]
        lib.ref3d_macroscopic.argtypes = [_vp, _dp, _dp, _dp, _dp]
        lib.ref3d_mass.argtypes = [_vp, _dp]
        lib.ref3d_link_count.argtypes = [_vp]
        lib.ref3d_link_count.restype = ctypes.c_uint64
        lib.ref3d_links.argtypes = [_vp, _u32p, _u32p, _dp]
        lib.ref3d_steps.argtypes = [_vp]
        lib.ref3d_steps.restype = ctypes.c_uint64
        lib.ref3d_sphere_mask.argtypes = [ctypes.c_uint64] * 3 + [_dp, ctypes.c_double, _u8p, _dp]
        lib.ref3d_box_mask.argtypes = [ctypes.c_uint64] * 3 + [_dp, _dp, _u8p, _dp]
        lib.ref3d_memory.argtypes = [c3, ctypes.c_uint64, ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64)]
        lib.ref2d_validate.argtypes = [c2, _u8p, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref2d_create.restype = _vp
        lib.ref2d_create.argtypes = [c2, _u8p, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref2d_destroy.argtypes = [_vp]
        lib.ref2d_initialize.argtypes = [_vp, _dp, _dp, _dp]
        lib.ref2d_step.argtypes = [_vp, ctypes.c_uint64]
        lib.ref2d_populations.argtypes = [_vp, _dp]
        lib.ref2d_force.argtypes = [_vp, _dp]
        lib.ref2d_macroscopic.argtypes = [_vp, _dp, _dp, _dp]
        lib.ref2d_mass.argtypes = [_vp, _dp]
        lib.ref2d_circle_mask.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, _u8p]
        _reference = lib
    return _reference


class _Base3D:
    q = 19

    def __init__(self, config, solid, distance=None):
        self.config = config
        self.cells = config.cells
        self.solid = np.ascontiguousarray(solid, dtype=np.uint8).reshape(-1)
        self.distance = None if distance is None else np.ascontiguousarray(distance, dtype=np.float64).reshape(-1)
        self._c = config.to_c()

    def macroscopic(self):
        out = [np.empty(self.cells) for _ in range(4)]
        self._macroscopic(*out)
        return out

    def populations(self):
        f = np.empty(self.q * self.cells)
        self._populations(f)
        return f

    def force(self):
        out = np.empty(6)
        self._force(out)
        return out


class Restated3D(_Base3D):
    """The C restatement (lo3_*)."""

    def __init__(self, config, solid, distance=None):
        super().__init__(config, solid, distance)
        self._lib = restated_lib()
        self._h = self._lib.lo3_create(ctypes.byref(self._c), _ptr(self.solid, _u8p),
                                       _ptr(self.distance, _dp))

    def close(self):
        if self._h:
            self._lib.lo3_destroy(self._h)
            self._h = None

    __del__ = close

    def initialize(self, rho=None, ux=None, uy=None, uz=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (rho, ux, uy, uz)]
        self._lib.lo3_initialize(self._h, *[_ptr(a, _dp) for a in arrs])

    def step(self, n):
        self._lib.lo3_step(self._h, int(n))

    def set_inlet_velocity(self, u):
        v = np.asarray(u, dtype=np.float64)
        self._lib.lo3_set_inlet(self._h, _ptr(v, _dp))

    def _macroscopic(self, *out):
        self._lib.lo3_macroscopic(self._h, *[_ptr(a, _dp) for a in out])

    def _populations(self, f):
        self._lib.lo3_populations(self._h, _ptr(f, _dp))

    def _force(self, out):
        self._lib.lo3_force(self._h, _ptr(out, _dp))

    def mass(self):
        return self._lib.lo3_mass(self._h)

    def links(self):
        n = self._lib.lo3_link_count(self._h)
        cell = np.empty(n, np.uint32)
        d = np.empty(n, np.uint32)
        q = np.empty(n)
        self._lib.lo3_links(self._h, _ptr(cell, _u32p), _ptr(d, _u32p), _ptr(q, _dp))
        return cell, d, q

    def boundary_count(self):
        return self._lib.lo3_boundary_count(self._h)


class Reference3D(_Base3D):
    """Orrery's CpuLbm3D, built from the reference sources (ref3d_*)."""

    def __init__(self, config, solid, distance=None):
        super().__init__(config, solid, distance)
        self._lib = reference_lib()
        msg = ctypes.create_string_buffer(1024)
        self._h = self._lib.ref3d_create(ctypes.byref(self._c), _ptr(self.solid, _u8p),
                                         _ptr(self.distance, _dp), msg, 1024)
        if not self._h:
            raise ValueError(msg.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ref3d_destroy(self._h)
            self._h = None

    __del__ = close

    def initialize(self, rho=None, ux=None, uy=None, uz=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (rho, ux, uy, uz)]
        if self._lib.ref3d_initialize(self._h, *[_ptr(a, _dp) for a in arrs]) != 0:
            raise RuntimeError("reference initialize failed")

    def step(self, n):
        if self._lib.ref3d_step(self._h, int(n)) != 0:
            raise RuntimeError("reference step failed")

    def set_inlet_velocity(self, u):
        v = np.asarray(u, dtype=np.float64)
        msg = ctypes.create_string_buffer(1024)
        if self._lib.ref3d_set_inlet(self._h, _ptr(v, _dp), msg, 1024) != 0:
            raise ValueError(msg.value.decode())

    def _macroscopic(self, *out):
        self._lib.ref3d_macroscopic(self._h, *[_ptr(a, _dp) for a in out])

    def _populations(self, f):
        self._lib.ref3d_populations(self._h, _ptr(f, _dp))

    def _force(self, out):
        self._lib.ref3d_force(self._h, _ptr(out, _dp))

    def mass(self):
        out = ctypes.c_double()
        self._lib.ref3d_mass(self._h, ctypes.byref(out))
        return out.value

    def links(self):
        n = self._lib.ref3d_link_count(self._h)
        cell = np.empty(n, np.uint32)
        d = np.empty(n, np.uint32)
        q = np.empty(n)
        self._lib.ref3d_links(self._h, _ptr(cell, _u32p), _ptr(d, _u32p), _ptr(q, _dp))
        return cell, d, q


def reference_validate3d(config, solid, distance=None):
    """The reference's validate() message ('' when accepted)."""
    lib = reference_lib()
    c = config.to_c()
    s = np.ascontiguousarray(solid, dtype=np.uint8).reshape(-1)
    d = None if distance is None else np.ascontiguousarray(distance, dtype=np.float64).reshape(-1)
    msg = ctypes.create_string_buffer(1024)
    lib.ref3d_validate(ctypes.byref(c), _ptr(s, _u8p), _ptr(d, _dp), msg, 1024)
    return msg.value.decode()


def reference_sphere_mask(nx, ny, nz, centre, radius):
    lib = reference_lib()
    n = nx * ny * nz
    solid = np.empty(n, np.uint8)
    dist = np.empty(n)
    c = np.asarray(centre, dtype=np.float64)
    lib.ref3d_sphere_mask(nx, ny, nz, _ptr(c, _dp), float(radius), _ptr(solid, _u8p), _ptr(dist, _dp))
    return solid, dist


def reference_box_mask(nx, ny, nz, lo, hi):
    lib = reference_lib()
    n = nx * ny * nz
    solid = np.empty(n, np.uint8)
    dist = np.empty(n)
    a = np.asarray(lo, dtype=np.float64)
    b = np.asarray(hi, dtype=np.float64)
    lib.ref3d_box_mask(nx, ny, nz, _ptr(a, _dp), _ptr(b, _dp), _ptr(solid, _u8p), _ptr(dist, _dp))
    return solid, dist


def reference_memory3d(config, links, wall_slots):
    lib = reference_lib()
    c = config.to_c()
    a, b, cpu = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    if lib.ref3d_memory(ctypes.byref(c), links, wall_slots, ctypes.byref(a), ctypes.byref(b),
                        ctypes.byref(cpu)) != 0:
        return None
    return a.value, b.value, cpu.value


class _Base2D:
    q = 9

    def __init__(self, config, solid):
        self.config = config
        self.cells = config.cells
        self.solid = np.ascontiguousarray(solid, dtype=np.uint8).reshape(-1)
        self._c = config.to_c()

    def macroscopic(self):
        out = [np.empty(self.cells) for _ in range(3)]
        self._macroscopic(*out)
        return out

    def populations(self):
        f = np.empty(self.q * self.cells)
        self._populations(f)
        return f

    def force(self):
        out = np.empty(3)
        self._force(out)
        return out


class Restated2D(_Base2D):
    def __init__(self, config, solid):
        super().__init__(config, solid)
        self._lib = restated_lib()
        self._h = self._lib.lo2_create(ctypes.byref(self._c), _ptr(self.solid, _u8p))

    def close(self):
        if self._h:
            self._lib.lo2_destroy(self._h)
            self._h = None

    __del__ = close

    def initialize(self, rho=None, ux=None, uy=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (rho, ux, uy)]
        self._lib.lo2_initialize(self._h, *[_ptr(a, _dp) for a in arrs])

    def step(self, n):
        self._lib.lo2_step(self._h, int(n))

    def _macroscopic(self, *out):
        self._lib.lo2_macroscopic(self._h, *[_ptr(a, _dp) for a in out])

    def _populations(self, f):
        self._lib.lo2_populations(self._h, _ptr(f, _dp))

    def _force(self, out):
        self._lib.lo2_force(self._h, _ptr(out, _dp))

    def mass(self):
        return self._lib.lo2_mass(self._h)

    def links(self):
        n = self._lib.lo2_link_count(self._h)
        cell = np.empty(n, np.uint32)
        d = np.empty(n, np.uint32)
        self._lib.lo2_links(self._h, _ptr(cell, _u32p), _ptr(d, _u32p))
        return cell, d


class Reference2D(_Base2D):
    def __init__(self, config, solid):
        super().__init__(config, solid)
        self._lib = reference_lib()
        msg = ctypes.create_string_buffer(1024)
        self._h = self._lib.ref2d_create(ctypes.byref(self._c), _ptr(self.solid, _u8p), msg, 1024)
        if not self._h:
            raise ValueError(msg.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ref2d_destroy(self._h)
            self._h = None

    __del__ = close

    def initialize(self, rho=None, ux=None, uy=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (rho, ux, uy)]
        self._lib.ref2d_initialize(self._h, *[_ptr(a, _dp) for a in arrs])

    def step(self, n):
        self._lib.ref2d_step(self._h, int(n))

    def _macroscopic(self, *out):
        self._lib.ref2d_macroscopic(self._h, *[_ptr(a, _dp) for a in out])

    def _populations(self, f):
        self._lib.ref2d_populations(self._h, _ptr(f, _dp))

    def _force(self, out):
        self._lib.ref2d_force(self._h, _ptr(out, _dp))

    def mass(self):
        out = ctypes.c_double()
        self._lib.ref2d_mass(self._h, ctypes.byref(out))
        return out.value


def reference_validate2d(config, solid):
    lib = reference_lib()
    c = config.to_c()
    s = np.ascontiguousarray(solid, dtype=np.uint8).reshape(-1)
    msg = ctypes.create_string_buffer(1024)
    lib.ref2d_validate(ctypes.byref(c), _ptr(s, _u8p), msg, 1024)
    return msg.value.decode()


def reference_circle_mask(nx, ny, cx, cy, radius):
    lib = reference_lib()
    solid = np.empty(nx * ny, np.uint8)
    lib.ref2d_circle_mask(nx, ny, float(cx), float(cy), float(radius), _ptr(solid, _u8p))
    return solid


def set_threads(n: int) -> None:
    restated_lib().lo_set_threads(int(n))
    if reference_available():
        reference_lib().ref_set_threads(int(n))


# ---- mesh voxelization (reference geom::voxelize, geom::signed_distance_band) ----

def _geom_lib():
    lib = reference_lib()
    if not getattr(lib, "_geom_declared", False):
        u64p = ctypes.POINTER(ctypes.c_uint64)
        cp, sz = ctypes.c_char_p, ctypes.c_size_t
        lib.ref_mesh_sphere.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_double, u64p, u64p, cp, sz]
        lib.ref_mesh_ellipsoid.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_double, u64p, u64p, cp, sz]
        lib.ref_mesh_cone.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, u64p, u64p, cp, sz]
        lib.ref_mesh_box.argtypes = [ctypes.c_double] * 3 + [u64p, u64p, cp, sz]
        lib.ref_mesh_naca_wing.argtypes = [cp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                           u64p, u64p, cp, sz]
        lib.ref_mesh_copy.argtypes = [_dp, _u32p]
        lib.ref_grid_around.argtypes = [_dp, _dp, ctypes.c_double, ctypes.c_uint64, _dp, u64p, cp, sz]
        lib.ref_voxelize.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp, ctypes.c_double,
                                     ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double, _u8p, _dp,
                                     cp, sz]
        lib.ref_signed_distance_band.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp,
                                                 ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.c_uint64, _u8p, ctypes.c_uint64, ctypes.c_double, _dp,
                                                 _u8p, _dp, cp, sz]
        lib.ref_winding_direct.restype = ctypes.c_double
        lib.ref_winding_direct.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp]
        lib.ref_solid_angle.restype = ctypes.c_double
        lib.ref_solid_angle.argtypes = [_dp, _dp, _dp, _dp]
        lib.ref_closest_point.argtypes = [_dp, _dp, _dp, _dp, _dp]
        lib.ref_hypot3.restype = ctypes.c_double
        lib.ref_hypot3.argtypes = [ctypes.c_double] * 3
        lib._geom_declared = True
    return lib


class ReferenceError_(RuntimeError):
    """A std::invalid_argument (or other exception) of the reference."""


def reference_mesh(kind: str, *args):
    """Vertices (n, 3) and triangles (m, 3) of a reference mesh builder:
    'sphere' (radius, around, arc_step), 'ellipsoid' (a, b, c, around,
    arc_step), 'cone' (radius, height, around), 'box' (lx, ly, lz),
    'naca_wing' (digits, chord, span, n, span_divisions)."""
    lib = _geom_lib()
    nv, nt = ctypes.c_uint64(), ctypes.c_uint64()
    msg = ctypes.create_string_buffer(1024)
    fn = getattr(lib, "ref_mesh_" + kind)
    if kind == "naca_wing":
        args = (args[0].encode(),) + tuple(args[1:])
    rc = fn(*args, ctypes.byref(nv), ctypes.byref(nt), msg, 1024)
    if rc != 0:
        raise ReferenceError_(msg.value.decode())
    v = np.empty((nv.value, 3), np.float64)
    t = np.empty((nt.value, 3), np.uint32)
    lib.ref_mesh_copy(_ptr(v, _dp), _ptr(t, _u32p))
    return v, t


def reference_grid_around(lo, hi, spacing, padding):
    lib = _geom_lib()
    lo = np.ascontiguousarray(lo, np.float64)
    hi = np.ascontiguousarray(hi, np.float64)
    origin = np.empty(3, np.float64)
    n = np.empty(3, np.uint64)
    msg = ctypes.create_string_buffer(1024)
    if lib.ref_grid_around(_ptr(lo, _dp), _ptr(hi, _dp), float(spacing), int(padding), _ptr(origin, _dp),
                           n.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), msg, 1024) != 0:
        raise ReferenceError_(msg.value.decode())
    return origin, [int(x) for x in n]


def reference_voxelize(vertices, triangles, origin, spacing, n, threshold=0.5):
    lib = _geom_lib()
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    o = np.ascontiguousarray(origin, np.float64)
    cells = int(n[0]) * int(n[1]) * int(n[2])
    cells = cells if 0 < cells <= (1 << 27) else 1   # refused grids are not written
    solid = np.zeros(cells, np.uint8)
    wind = np.zeros(cells, np.float64)
    msg = ctypes.create_string_buffer(1024)
    if lib.ref_voxelize(_ptr(v, _dp), len(v), _ptr(t, _u32p), len(t), _ptr(o, _dp), float(spacing), int(n[0]),
                        int(n[1]), int(n[2]), float(threshold), _ptr(solid, _u8p), _ptr(wind, _dp), msg, 1024) != 0:
        raise ReferenceError_(msg.value.decode())
    return solid, wind


def reference_signed_distance_band(vertices, triangles, origin, spacing, n, solid, band_cells=3.0):
    lib = _geom_lib()
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    o = np.ascontiguousarray(origin, np.float64)
    s = np.ascontiguousarray(solid, np.uint8)
    cells = max(len(s), 1)
    dist = np.zeros(cells, np.float64)
    inb = np.zeros(cells, np.uint8)
    band = ctypes.c_double()
    msg = ctypes.create_string_buffer(1024)
    if lib.ref_signed_distance_band(_ptr(v, _dp), len(v), _ptr(t, _u32p), len(t), _ptr(o, _dp), float(spacing),
                                    int(n[0]), int(n[1]), int(n[2]), _ptr(s, _u8p), len(s), float(band_cells),
                                    _ptr(dist, _dp), _ptr(inb, _u8p), ctypes.byref(band), msg, 1024) != 0:
        raise ReferenceError_(msg.value.decode())
    return dist[:len(s)], inb[:len(s)], band.value


# ---- the reference's 3D adapter (LbmAeroSolver3D), CPU solver or CUDA solver ----

ADAPTER_SO = os.path.join(os.path.dirname(REFERENCE_SO), "libref_adapter.so")
ADAPTER_VOXEL_SO = os.path.join(os.path.dirname(REFERENCE_SO), "libref_adapter_voxel.so")
_adapter = {}

ADAPTER_DEFAULTS = {
    "length": 1.0, "area": 1.0, "speed": 1.0, "density": 1.225, "viscosity": 1.789e-5,
    "angle_of_attack": 0.0, "sideslip": 0.0, "cells_per_length": 16.0, "lattice_velocity": 0.05,
    "upstream": 5.0, "downstream": 10.0, "width": 6.0, "duration": 30.0, "average_window": 8.0,
    "steps_per_call": 200, "wall": 1, "sponge_strength": 0.1, "start_ramp": 3.0, "les": 0, "sample_every": 10,
}
_ADAPTER_ORDER = ["length", "area", "speed", "density", "viscosity", "angle_of_attack", "sideslip",
                  "cells_per_length", "lattice_velocity", "upstream", "downstream", "width", "duration",
                  "average_window", "steps_per_call", "wall", "sponge_strength", "start_ramp", "les", "sample_every"]
_ADAPTER_OUT = ["cd", "cl", "cy", "cm", "fx", "fy", "fz", "mx", "my", "mz", "iterations", "converged", "seconds",
                "nx", "ny", "nz", "lattice_steps"]


def adapter_available() -> bool:
    return os.path.exists(ADAPTER_SO) and os.path.exists(ADAPTER_VOXEL_SO)


def reference_adapter_run(vertices, triangles, backend: str = "cpu", storage: int = 0, voxelizer: str = "cpu",
                          fields: bool = False, **params) -> dict:
    """One LbmAeroSolver3D solve (setup, then step() until done) of the
    reference's own adapter; backend 'cpu' is its CPU solver, 'cuda' the CUDA
    solver through the Lbm3DSolver seam (ORR_STORAGE_* `storage`); voxelizer
    'cpu' is the reference's geom::voxelize, 'device' the drop-in of
    orrery_b200/adapter/voxel_grid_cuda.cpp.  fields: also the result's wall
    pressure coefficients ("cp") and velocity field ("velocity", m/s, n x 3)."""
    path = ADAPTER_VOXEL_SO if voxelizer == "device" else ADAPTER_SO
    if path not in _adapter:
        lib = ctypes.CDLL(path)
        lib.ref_adapter_run.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp, ctypes.c_int,
                                        ctypes.c_int, _dp, ctypes.c_char_p, ctypes.c_size_t]
        _adapter[path] = lib
    lib = _adapter[path]
    p = dict(ADAPTER_DEFAULTS)
    p.update(params)
    arr = np.array([float(p[k]) for k in _ADAPTER_ORDER])
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    out = np.zeros(len(_ADAPTER_OUT))
    msg = ctypes.create_string_buffer(2048)
    rc = lib.ref_adapter_run(_ptr(v, _dp), len(v), _ptr(t, _u32p), len(t), _ptr(arr, _dp),
                                  1 if backend == "cuda" else 0, int(storage), _ptr(out, _dp), msg, 2048)
    if rc != 0:
        raise ReferenceError_(msg.value.decode())
    result = dict(zip(_ADAPTER_OUT, out.tolist()))
    if fields:
        u64 = ctypes.POINTER(ctypes.c_uint64)
        lib.ref_adapter_fields.argtypes = [u64, u64, _dp, _dp]
        nc, nv_ = ctypes.c_uint64(), ctypes.c_uint64()
        lib.ref_adapter_fields(ctypes.byref(nc), ctypes.byref(nv_), None, None)
        cp = np.zeros(max(nc.value, 1))
        vel = np.zeros(max(nv_.value, 1))
        lib.ref_adapter_fields(ctypes.byref(nc), ctypes.byref(nv_), _ptr(cp, _dp), _ptr(vel, _dp))
        result["cp"] = cp[:nc.value]
        result["velocity"] = vel[:nv_.value].reshape(-1, 3)
    return result


def _adapter_lib():
    if ADAPTER_SO not in _adapter:
        lib = ctypes.CDLL(ADAPTER_SO)
        lib.ref_adapter_run.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp, ctypes.c_int,
                                        ctypes.c_int, _dp, ctypes.c_char_p, ctypes.c_size_t]
        _adapter[ADAPTER_SO] = lib
    lib = _adapter[ADAPTER_SO]
    lib.ref_cd_table.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp, ctypes.c_double, _dp,
                                 ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _dp, ctypes.c_char_p,
                                 ctypes.c_size_t]
    lib.ref_cd_point_problem.argtypes = [_dp, ctypes.c_uint64, _u32p, ctypes.c_uint64, _dp, ctypes.c_double,
                                         ctypes.c_double, ctypes.POINTER(abi.CLbm3DConfig), _u8p, _dp, _dp,
                                         ctypes.c_char_p, ctypes.c_size_t]
    return lib


_TABLE_OUT = ["mach", "cd", "solver_steps", "converged", "within_envelope", "seconds", "table_cd", "table_seconds"]


def reference_cd_table(vertices, triangles, mach, temperature: float = 288.15, max_steps: int = 100000,
                       storage: int = 0, **params) -> list[dict]:
    """The reference's atmo::sample_cd_table (src/atmo/cd_sampling.cpp:98-120)
    with the lattice Boltzmann solver forced and a factory of the reference's
    LbmAeroSolver3D on the CUDA solver (ORR_STORAGE_* `storage`): one adapter
    solve per Mach number, one after another.  `params` as for
    reference_adapter_run (the speed is Mach times the speed of sound of
    `temperature`).  One dict per point."""
    lib = _adapter_lib()
    p = dict(ADAPTER_DEFAULTS)
    p.update(params)
    arr = np.array([float(p[k]) for k in _ADAPTER_ORDER])
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    m = np.ascontiguousarray(mach, np.float64)
    out = np.zeros(len(m) * len(_TABLE_OUT))
    msg = ctypes.create_string_buffer(2048)
    if lib.ref_cd_table(_ptr(v, _dp), len(v), _ptr(t, _u32p), len(t), _ptr(arr, _dp), float(temperature),
                        _ptr(m, _dp), len(m), int(max_steps), int(storage), _ptr(out, _dp), msg, 2048) != 0:
        raise ReferenceError_(msg.value.decode())
    return [dict(zip(_TABLE_OUT, row.tolist())) for row in out.reshape(len(m), len(_TABLE_OUT))]


_PROBLEM_META = ["nx", "ny", "nz", "total_steps", "window_samples", "ramp_steps", "dx", "area_lattice",
                 "length_lattice", "lattice_velocity", "sample_every", "has_distance"]


def reference_cd_point_problem(vertices, triangles, mach: float, temperature: float = 288.15, **params) -> dict:
    """The lattice problem the reference adapter's setup builds for one Mach
    point of reference_cd_table: "config" (abi.CLbm3DConfig), "solid",
    "distance" (or None), and the run lengths and lattice reference values of
    _PROBLEM_META."""
    lib = _adapter_lib()
    p = dict(ADAPTER_DEFAULTS)
    p.update(params)
    arr = np.array([float(p[k]) for k in _ADAPTER_ORDER])
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    cfg = abi.CLbm3DConfig()
    meta = np.zeros(len(_PROBLEM_META))
    msg = ctypes.create_string_buffer(2048)
    args = (_ptr(v, _dp), len(v), _ptr(t, _u32p), len(t), _ptr(arr, _dp), float(temperature), float(mach),
            ctypes.byref(cfg))
    if lib.ref_cd_point_problem(*args, None, None, _ptr(meta, _dp), msg, 2048) != 0:
        raise ReferenceError_(msg.value.decode())
    cells = int(meta[0]) * int(meta[1]) * int(meta[2])
    solid = np.zeros(cells, np.uint8)
    dist = np.zeros(cells) if meta[11] else None
    if lib.ref_cd_point_problem(*args, _ptr(solid, _u8p), _ptr(dist, _dp), _ptr(meta, _dp), msg, 2048) != 0:
        raise ReferenceError_(msg.value.decode())
    out = dict(zip(_PROBLEM_META, meta.tolist()))
    out.update({"config": cfg, "solid": solid, "distance": dist})
    return out


def reference_cd_lookup(samples, query, area: float = 1.0):
    """The reference's AeroCoefficientTable::create + lookup
    (src/atmo/aero_table.cpp:47-83): (cd, clamped) at every query Mach, or
    ReferenceError_ with the refusal's text."""
    lib = _adapter_lib()
    lib.ref_cd_table_lookup.argtypes = [_dp, _dp, ctypes.c_uint64, ctypes.c_double, _dp, ctypes.c_uint64, _dp,
                                        _u8p, ctypes.c_char_p, ctypes.c_size_t]
    m = np.ascontiguousarray([s[0] for s in samples], np.float64)
    c = np.ascontiguousarray([s[1] for s in samples], np.float64)
    q = np.ascontiguousarray(query, np.float64)
    out = np.zeros(max(len(q), 1))
    clamped = np.zeros(max(len(q), 1), np.uint8)
    msg = ctypes.create_string_buffer(1024)
    if lib.ref_cd_table_lookup(_ptr(m, _dp), _ptr(c, _dp), len(m), float(area), _ptr(q, _dp),
                               len(q), _ptr(out, _dp), _ptr(clamped, _u8p), msg, 1024) != 0:
        raise ReferenceError_(msg.value.decode())
    return out[:len(q)], clamped[:len(q)].astype(bool)


# ---- the reference's GPU driver (GpuLbm3D) on the CUDA compute backend ----

BACKEND_SO = os.path.join(os.path.dirname(REFERENCE_SO), "libref_backend.so")
_backend = None


def backend_available() -> bool:
    return os.path.exists(BACKEND_SO)


def _backend_lib():
    global _backend
    if _backend is None:
        lib = ctypes.CDLL(BACKEND_SO)
        lib.ref_backend_solve.argtypes = [ctypes.POINTER(abi.CLbm3DConfig), _u8p, _dp, _dp, _dp, _dp, _dp,
                                          ctypes.c_uint64, _dp, _dp, _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_backend_solve2d.argtypes = [ctypes.POINTER(abi.CLbm2DConfig), _u8p, _dp, _dp, _dp,
                                            ctypes.c_uint64, _dp, _dp, _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_backend_refusals.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_backend_adapter2d.argtypes = [_dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_cuda2d_solve.argtypes = [ctypes.POINTER(abi.CLbm2DConfig), _u8p, _dp, _dp, _dp, ctypes.c_uint64,
                                         _dp, _dp, _dp, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_backend_adapter3d.argtypes = [_dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_backend_rate3d.argtypes = [ctypes.POINTER(abi.CLbm3DConfig), _u8p, ctypes.c_uint64,
                                           ctypes.c_uint64, _dp, ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_backend_rate2d.argtypes = [ctypes.POINTER(abi.CLbm2DConfig), _u8p, ctypes.c_uint64,
                                           ctypes.c_uint64, _dp, ctypes.c_char_p, ctypes.c_size_t]
        _backend = lib
    return _backend


def reference_gpu_driver_solve(config, solid, distance=None, fields=None, steps: int = 0) -> dict:
    """One solve of the reference's own GPU driver (make_gpu_solver of
    src/aero/lbm3d/lbm3d_gpu.cpp) on the CUDA compute backend: initial fields
    (rho, ux, uy, uz) or the uniform inlet state, `steps` steps; returns the
    populations, the moments (density, ux, uy, uz), force and moment, and the
    backend's dispatch count and node-code tables built."""
    lib = _backend_lib()
    c = config.to_c()
    n = config.cells
    s = np.ascontiguousarray(solid, np.uint8).reshape(-1)
    d = None if distance is None else np.ascontiguousarray(distance, np.float64).reshape(-1)
    f = [None] * 4 if fields is None else [np.ascontiguousarray(a, np.float64).reshape(-1) for a in fields]
    pops = np.zeros(19 * n)
    mom = np.zeros(4 * n)
    force = np.zeros(6)
    meta = np.zeros(4)
    msg = ctypes.create_string_buffer(2048)
    rc = lib.ref_backend_solve(ctypes.byref(c), _ptr(s, _u8p), _ptr(d, _dp), *[_ptr(a, _dp) for a in f],
                               int(steps), _ptr(pops, _dp), _ptr(mom, _dp), _ptr(force, _dp), _ptr(meta, _dp),
                               msg, 2048)
    if rc != 0:
        raise ReferenceError_(msg.value.decode())
    return {"populations": pops, "density": mom[:n], "ux": mom[n:2 * n], "uy": mom[2 * n:3 * n],
            "uz": mom[3 * n:], "force": force[:3], "moment": force[3:], "dispatches": int(meta[0]),
            "tables_built": int(meta[1]), "executes_kernels": bool(meta[2]), "steps": int(meta[3])}


def reference_gpu_driver_solve2d(config, solid, fields=None, steps: int = 0) -> dict:
    """One solve of the reference's own D2Q9 GPU driver (make_gpu_solver of
    src/aero/lbm/lbm2d_gpu.cpp) on the CUDA compute backend: initial fields
    (rho, ux, uy) or the uniform inlet state, `steps` steps; returns the
    populations, the moments (density, ux, uy), the force (x, y, moment) and
    the backend's dispatch count and solid-flag tables built."""
    lib = _backend_lib()
    c = config.to_c()
    n = int(config.nx) * int(config.ny)
    s = np.ascontiguousarray(solid, np.uint8).reshape(-1)
    f = [None] * 3 if fields is None else [np.ascontiguousarray(a, np.float64).reshape(-1) for a in fields]
    pops = np.zeros(9 * n)
    mom = np.zeros(3 * n)
    force = np.zeros(3)
    meta = np.zeros(4)
    msg = ctypes.create_string_buffer(2048)
    rc = lib.ref_backend_solve2d(ctypes.byref(c), _ptr(s, _u8p), *[_ptr(a, _dp) for a in f], int(steps),
                                 _ptr(pops, _dp), _ptr(mom, _dp), _ptr(force, _dp), _ptr(meta, _dp), msg, 2048)
    if rc != 0:
        raise ReferenceError_(msg.value.decode())
    return {"populations": pops, "density": mom[:n], "ux": mom[n:2 * n], "uy": mom[2 * n:], "force": force,
            "dispatches": int(meta[0]), "tables_built": int(meta[1]), "executes_kernels": bool(meta[2]),
            "steps": int(meta[3])}


def reference_cuda2d_solve(config, solid, fields=None, steps: int = 0) -> dict:
    """One solve through the Lbm2DSolver seam: make_cuda_solver of
    orrery_b200/adapter/lbm2d_cuda.cpp (the C++ adapter over the C ABI),
    compiled against the reference's headers; outputs as
    reference_gpu_driver_solve2d."""
    lib = _backend_lib()
    c = config.to_c()
    n = int(config.nx) * int(config.ny)
    s = np.ascontiguousarray(solid, np.uint8).reshape(-1)
    f = [None] * 3 if fields is None else [np.ascontiguousarray(a, np.float64).reshape(-1) for a in fields]
    pops = np.zeros(9 * n)
    mom = np.zeros(3 * n)
    force = np.zeros(3)
    meta = np.zeros(1)
    msg = ctypes.create_string_buffer(2048)
    rc = lib.ref_cuda2d_solve(ctypes.byref(c), _ptr(s, _u8p), *[_ptr(a, _dp) for a in f], int(steps),
                              _ptr(pops, _dp), _ptr(mom, _dp), _ptr(force, _dp), _ptr(meta, _dp), msg, 2048)
    if rc != 0:
        raise ReferenceError_(msg.value.decode())
    return {"populations": pops, "density": mom[:n], "ux": mom[n:2 * n], "uy": mom[2 * n:], "force": force,
            "steps": int(meta[0])}


def reference_adapter2d_on_backend() -> dict:
    """The reference's 2D adapter (LbmAeroSolver2D) on its CPU solver and on
    the GPU driver over the CUDA backend, the case of the reference's
    "IAeroSolver adapter runs on the GPU backend" test."""
    out = np.zeros(6)
    msg = ctypes.create_string_buffer(2048)
    if _backend_lib().ref_backend_adapter2d(_ptr(out, _dp), msg, 2048) != 0:
        raise ReferenceError_(msg.value.decode())
    return {"cd_cpu": float(out[0]), "cd_gpu": float(out[1]), "iterations_cpu": int(out[2]),
            "iterations_gpu": int(out[3]), "cp_cpu": int(out[4]), "cp_gpu": int(out[5])}


def reference_adapter3d_on_backend() -> dict:
    """The reference's 3D adapter (LbmAeroSolver3D) on its CPU solver and on
    its own GPU driver over the CUDA backend, the case of the reference's
    "3D IAeroSolver adapter runs on the GPU backend" test."""
    out = np.zeros(4)
    msg = ctypes.create_string_buffer(2048)
    if _backend_lib().ref_backend_adapter3d(_ptr(out, _dp), msg, 2048) != 0:
        raise ReferenceError_(msg.value.decode())
    return {"cd_cpu": float(out[0]), "cd_gpu": float(out[1]), "iterations_cpu": int(out[2]),
            "iterations_gpu": int(out[3])}


def reference_driver_rate(config, solid, warmup: int = 50, count: int = 1000) -> float:
    """Steps per second of the reference's own GPU benchmark loop with its GPU
    driver (3D or 2D, by the configuration) on the CUDA backend."""
    lib = _backend_lib()
    c = config.to_c()
    s = np.ascontiguousarray(solid, np.uint8).reshape(-1)
    seconds = np.zeros(1)
    msg = ctypes.create_string_buffer(2048)
    fn = lib.ref_backend_rate3d if isinstance(c, abi.CLbm3DConfig) else lib.ref_backend_rate2d
    if fn(ctypes.byref(c), _ptr(s, _u8p), int(warmup), int(count), _ptr(seconds, _dp), msg, 2048) != 0:
        raise ReferenceError_(msg.value.decode())
    return count / float(seconds[0])


def reference_backend_refusals():
    """(refusals of the CUDA backend's five bad calls, the last refusal's text)."""
    msg = ctypes.create_string_buffer(1024)
    n = _backend_lib().ref_backend_refusals(msg, 1024)
    return n, msg.value.decode()


# ---- binary32 restatement of the reference's GPU step (GLSL kernels) ----

RESTATED32_SO = os.path.join(HERE, "_build", "liblbm_oracle32.so")
_restated32 = None


def restated32_lib():
    global _restated32
    if _restated32 is None:
        if not os.path.exists(RESTATED32_SO):
            build()
        lib = ctypes.CDLL(RESTATED32_SO)
        _fp = ctypes.POINTER(ctypes.c_float)
        lib.lo32_create.restype = _vp
        lib.lo32_create.argtypes = [ctypes.POINTER(abi.CLbm3DConfig), _u8p, _fp]
        lib.lo32_destroy.argtypes = [_vp]
        lib.lo32_initialize.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp]
        lib.lo32_set_inlet.argtypes = [_vp, _dp]
        lib.lo32_step.argtypes = [_vp, ctypes.c_uint64]
        lib.lo32_populations.argtypes = [_vp, _dp]
        lib.lo32_force.argtypes = [_vp, _u32p, _u32p, _dp, ctypes.c_uint64, _dp]
        lib.lo32_steps.restype = ctypes.c_uint64
        lib.lo32_steps.argtypes = [_vp]
        _restated32 = lib
    return _restated32


class Restated32:
    """The binary32 restatement of the reference's GLSL step
    (oracle/lbm_oracle32.c).  `links` are the lattice's boundary links (cell,
    direction, q), from the reference planner; their fractions fill the wall
    table of an interpolated wall."""

    def __init__(self, config, solid, links):
        self.lib = restated32_lib()
        self.config = config
        self.cells = config.cells
        self._c = config.to_c()
        self.solid = np.ascontiguousarray(solid, np.uint8).reshape(-1)
        cell, direction, q = links
        self.cell = np.ascontiguousarray(cell, np.uint32)
        self.direction = np.ascontiguousarray(direction, np.uint32)
        self.q = np.ascontiguousarray(q, np.float64)
        wall = None
        if int(config.solid_wall) == abi.ORR_SOLID_INTERPOLATED:
            wall = np.full(19 * self.cells, 0.5, np.float32)
            wall[self.cell.astype(np.int64) * 19 + self.direction] = self.q.astype(np.float32)
        self._wall = wall
        self.h = self.lib.lo32_create(ctypes.byref(self._c), _ptr(self.solid, _u8p),
                                      None if wall is None else wall.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        if not self.h:
            raise MemoryError("lo32_create")

    def close(self):
        if self.h:
            self.lib.lo32_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def initialize(self, rho=None, ux=None, uy=None, uz=None):
        c = self.config
        n = self.cells
        inflow = int(c.x_boundary) == abi.ORR_X_INFLOW_OUTFLOW
        if rho is None:
            rho = np.ones(n)
            ux = np.full(n, c.inlet_ux if inflow else 0.0)
            uy = np.full(n, c.inlet_uy if inflow else 0.0)
            uz = np.full(n, c.inlet_uz if inflow else 0.0)
        arrs = [np.ascontiguousarray(a, np.float64).reshape(-1) for a in (rho, ux, uy, uz)]
        inlet = np.array([c.inlet_ux, c.inlet_uy, c.inlet_uz], np.float64)
        self.lib.lo32_initialize(self.h, *[_ptr(a, _dp) for a in arrs], _ptr(inlet, _dp))

    def step(self, n):
        self.lib.lo32_step(self.h, int(n))

    def set_inlet_velocity(self, u):
        v = np.ascontiguousarray(u, np.float64)
        self.lib.lo32_set_inlet(self.h, _ptr(v, _dp))

    def populations(self):
        f = np.empty(19 * self.cells)
        self.lib.lo32_populations(self.h, _ptr(f, _dp))
        return f

    def force(self):
        out = np.empty(6)
        self.lib.lo32_force(self.h, _ptr(self.cell, _u32p), _ptr(self.direction, _u32p), _ptr(self.q, _dp),
                            len(self.cell), _ptr(out, _dp))
        return out
