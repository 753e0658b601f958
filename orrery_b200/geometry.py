"""Mesh voxelization on the device: solid masks and wall distances.

Mirrors the reference's geometry calls that build a lattice's mask
(src/geom/include/orrery/geom/voxel_grid.h):

    GridSpec                 geom::GridSpec
    grid_around(...)         geom::grid_around
    voxelize(mesh, spec)     geom::voxelize          -> VoxelGrid(spec, solid, winding)
    signed_distance_band()   geom::signed_distance_band -> SignedDistanceField

through orr_grid_around / orr_voxelize / orr_signed_distance_band of the
native library (generalized winding number and closest-triangle distance,
one device thread per cell).  Refusals raise ``LbmError`` with the
reference's texts.

The mesh builders here (solids of revolution such as the sphere-cone bodies
of the served workload, and boxes) are this package's own; meshes use the
reference's convention: counter-clockwise triangles seen from outside.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import abi
from ._native import LbmError, check, lib, ptr

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)


@dataclass
class TriangleMesh:
    """geom::TriangleMesh: vertices (n, 3) float64, triangles (m, 3) uint32."""
    vertices: np.ndarray
    triangles: np.ndarray

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float64).reshape(-1, 3)
        self.triangles = np.ascontiguousarray(self.triangles, dtype=np.uint32).reshape(-1, 3)

    def bounds(self):
        if len(self.vertices) == 0:
            return np.zeros(3), np.zeros(3)
        return self.vertices.min(axis=0), self.vertices.max(axis=0)

    def _c(self) -> abi.CMesh:
        m = abi.CMesh()
        m.vertices = ptr(self.vertices, _dp)
        m.vertex_count = len(self.vertices)
        m.triangles = ptr(self.triangles, _u32p)
        m.triangle_count = len(self.triangles)
        return m


@dataclass
class GridSpec:
    """geom::GridSpec: cell (i, j, k) has its centre at origin + spacing (i + 1/2,
    j + 1/2, k + 1/2) and index i + nx (j + ny k)."""
    origin: tuple
    spacing: float
    nx: int
    ny: int
    nz: int

    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def centre(self, i, j, k):
        o = self.origin
        h = self.spacing
        return (o[0] + (i + 0.5) * h, o[1] + (j + 0.5) * h, o[2] + (k + 0.5) * h)

    def _c(self) -> abi.CGridSpec:
        s = abi.CGridSpec()
        for k in range(3):
            s.origin[k] = float(self.origin[k])
        s.spacing = float(self.spacing)
        s.nx, s.ny, s.nz = int(self.nx), int(self.ny), int(self.nz)
        return s


@dataclass
class VoxelGrid:
    """geom::VoxelGrid: solid flags and winding numbers, x fastest."""
    spec: GridSpec
    solid: np.ndarray
    winding: np.ndarray | None
    device_ms: float = 0.0

    def solid_count(self) -> int:
        return int(np.count_nonzero(self.solid == 1))

    def mask(self) -> np.ndarray:
        """The solid flags as an (nz, ny, nx) array."""
        return self.solid.reshape(self.spec.nz, self.spec.ny, self.spec.nx)


@dataclass
class SignedDistanceField:
    """geom::SignedDistanceField: distance (negative inside) within `band`."""
    spec: GridSpec
    band: float
    distance: np.ndarray
    in_band: np.ndarray
    device_ms: float = 0.0


def _global_error():
    return lib().orr_last_error()


def grid_around(box_min, box_max, spacing: float, padding: int) -> GridSpec:
    lo = np.ascontiguousarray(box_min, dtype=np.float64)
    hi = np.ascontiguousarray(box_max, dtype=np.float64)
    out = abi.CGridSpec()
    check(lib().orr_grid_around(ptr(lo, _dp), ptr(hi, _dp), float(spacing), int(padding), ctypes.byref(out)),
          _global_error)
    return GridSpec(tuple(out.origin), out.spacing, out.nx, out.ny, out.nz)


def voxelize(mesh: TriangleMesh, spec: GridSpec, threshold: float = 0.5, device: int = 0,
             winding: bool = True) -> VoxelGrid:
    """Solid flags (winding number at the cell centre >= threshold) of every cell."""
    n = spec.cells() if spec.nx > 0 and spec.ny > 0 and spec.nz > 0 else 0
    if n > (1 << 27):
        n = 0   # refused by the library before anything is written
    solid = np.zeros(max(n, 1), dtype=np.uint8)
    wind = np.zeros(max(n, 1), dtype=np.float64) if winding else None
    ms = ctypes.c_double(0.0)
    c_mesh, c_spec = mesh._c(), spec._c()
    check(lib().orr_voxelize(ctypes.byref(c_mesh), ctypes.byref(c_spec), float(threshold), int(device),
                             ptr(solid, _u8p), ptr(wind, _dp), ctypes.byref(ms)), _global_error)
    return VoxelGrid(spec, solid[:n], None if wind is None else wind[:n], ms.value)


def signed_distance_band(mesh: TriangleMesh, voxels: VoxelGrid, band_cells: float = 3.0,
                         device: int = 0) -> SignedDistanceField:
    spec = voxels.spec
    solid = np.ascontiguousarray(voxels.solid, dtype=np.uint8)
    n = len(solid)
    distance = np.zeros(max(n, 1), dtype=np.float64)
    in_band = np.zeros(max(n, 1), dtype=np.uint8)
    band = ctypes.c_double(0.0)
    ms = ctypes.c_double(0.0)
    c_mesh, c_spec = mesh._c(), spec._c()
    check(lib().orr_signed_distance_band(ctypes.byref(c_mesh), ctypes.byref(c_spec), ptr(solid, _u8p), n,
                                         float(band_cells), int(device), ptr(distance, _dp), ptr(in_band, _u8p),
                                         ctypes.byref(band), ctypes.byref(ms)), _global_error)
    return SignedDistanceField(spec, band.value, distance[:n], in_band[:n], ms.value)


# ------------------------------------------------------------ mesh builders --

def revolution_mesh(profile, around: int) -> TriangleMesh:
    """Closed, outward mesh of a solid of revolution about z: `profile` is a
    list of (r, z) from a point on the axis (bottom) to a point on the axis
    (top), interior points off the axis; `around` vertices per ring."""
    pts = [(float(r), float(z)) for r, z in profile]
    if len(pts) < 3 or pts[0][0] != 0.0 or pts[-1][0] != 0.0 or any(r <= 0.0 for r, _ in pts[1:-1]):
        raise ValueError("profile must run from the axis to the axis through points off it")
    if around < 3:
        raise ValueError("around must be at least 3")
    ang = 2.0 * np.pi * np.arange(around) / around
    rings = pts[1:-1]
    verts = [(0.0, 0.0, pts[0][1])]
    for r, z in rings:
        verts.extend(zip(r * np.cos(ang), r * np.sin(ang), np.full(around, z)))
    top = len(verts)
    verts.append((0.0, 0.0, pts[-1][1]))
    tris = []
    ring = lambda k, j: 1 + k * around + (j % around)   # noqa: E731
    for j in range(around):
        tris.append((0, ring(0, j + 1), ring(0, j)))
    for k in range(len(rings) - 1):
        for j in range(around):
            a0, a1, b0, b1 = ring(k, j), ring(k, j + 1), ring(k + 1, j), ring(k + 1, j + 1)
            tris.append((a0, a1, b1))
            tris.append((a0, b1, b0))
    last = len(rings) - 1
    for j in range(around):
        tris.append((top, ring(last, j), ring(last, j + 1)))
    return TriangleMesh(np.array(verts), np.array(tris))


def sphere_mesh(radius: float, around: int = 64, rings: int = 31) -> TriangleMesh:
    phi = -0.5 * np.pi + np.pi * np.arange(1, rings + 1) / (rings + 1)
    prof = [(0.0, -radius)] + [(radius * np.cos(p), radius * np.sin(p)) for p in phi] + [(0.0, radius)]
    return revolution_mesh(prof, around)


def sphere_cone_mesh(base_radius: float, half_angle: float, nose_radius: float, around: int = 64,
                     nose_steps: int = 16, cone_steps: int = 16, axis: str = "x") -> TriangleMesh:
    """Sphere-cone: a spherical nose of `nose_radius` (tip at the origin), a cone
    of `half_angle` (radians) tangent to it out to `base_radius`, a flat base.
    The axis runs from the tip towards +x (or +z with axis='z')."""
    if not (0.0 < half_angle < 0.5 * np.pi) or not (0.0 < nose_radius) or not (base_radius > nose_radius * math.cos(half_angle)):
        raise ValueError("sphere-cone: invalid shape")
    polar_end = 0.5 * np.pi - half_angle
    prof = [(0.0, 0.0)]
    for p in polar_end * np.arange(1, nose_steps + 1) / nose_steps:
        prof.append((nose_radius * np.sin(p), nose_radius * (1.0 - np.cos(p))))
    rt, zt = prof[-1]
    zb = zt + (base_radius - rt) / math.tan(half_angle)
    for t in np.arange(1, cone_steps + 1) / cone_steps:
        prof.append((rt + t * (base_radius - rt), zt + t * (zb - zt)))
    prof.append((0.0, zb))
    m = revolution_mesh(prof, around)
    if axis == "x":
        v = m.vertices
        m = TriangleMesh(np.stack([v[:, 2], v[:, 0], v[:, 1]], axis=1), m.triangles)   # a rotation
    return m


def box_mesh(lx: float, ly: float, lz: float) -> TriangleMesh:
    hx, hy, hz = 0.5 * lx, 0.5 * ly, 0.5 * lz
    v = np.array([[x, y, z] for z in (-hz, hz) for y in (-hy, hy) for x in (-hx, hx)])
    # corner index = ix + 2 iy + 4 iz; two outward triangles per face
    t = [(0, 2, 3), (0, 3, 1), (4, 5, 7), (4, 7, 6),          # z- , z+
         (0, 1, 5), (0, 5, 4), (2, 6, 7), (2, 7, 3),          # y- , y+
         (0, 4, 6), (0, 6, 2), (1, 3, 7), (1, 7, 5)]          # x- , x+
    return TriangleMesh(v, np.array(t))
