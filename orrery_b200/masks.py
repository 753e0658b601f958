"""Solid masks for the lattices: flags plus the signed wall distance.

Restates the reference's mask builders with numpy so that a mask made here
is bit-for-bit the mask the reference builds:
``mask_from_sdf_3d``/``sphere_mask``/``box_mask``
(src/aero/lbm3d/solid_mask3d.cpp:57-102) and ``mask_from_sdf``/``circle_mask``
(src/aero/lbm/solid_mask.cpp:26-43).  A node (x, y, z) is solid where the
signed distance at its lattice position is <= 0; the distance is kept for the
interpolated wall.  Arrays are flat in the lattice order x + nx (y + ny z).

The body shapes of the benchmark workloads (prolate ellipsoid, NACA 4-digit
wing, sphere-cone capsule) are analytic signed distances evaluated the same way.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

MAX_GRID_CELLS = 1 << 27  # geom::max_grid_cells (src/geom/include/orrery/geom/voxel_grid.h:29)


@dataclass
class SolidMask3D:
    """SolidMask3D (src/aero/lbm3d/include/orrery/aero/lbm3d/solid_mask3d.h:28-44)."""
    nx: int
    ny: int
    nz: int
    solid: np.ndarray            # uint8, 1 solid / 0 fluid
    distance: np.ndarray | None  # float64 signed distance, or None

    def index(self, x: int, y: int, z: int) -> int:
        return x + self.nx * (y + self.ny * z)

    def count(self) -> int:
        return int(np.count_nonzero(self.solid))


@dataclass
class SolidMask2D:
    """SolidMask2D (src/aero/lbm/include/orrery/aero/lbm/solid_mask.h:19-28)."""
    nx: int
    ny: int
    solid: np.ndarray

    def count(self) -> int:
        return int(np.count_nonzero(self.solid))


def _grid3(nx: int, ny: int, nz: int):
    if nx <= 0 or ny <= 0 or nz <= 0 or nx * ny * nz > MAX_GRID_CELLS:
        raise ValueError("lbm3d: mask dimensions must be positive with at most "
                         "geom::max_grid_cells nodes")
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    return x.reshape(-1), y.reshape(-1), z.reshape(-1)


def fluid_mask_3d(nx: int, ny: int, nz: int) -> SolidMask3D:
    """fluid_mask_3d (solid_mask3d.cpp:43-55)."""
    if nx <= 0 or ny <= 0 or nz <= 0 or nx * ny * nz > MAX_GRID_CELLS:
        raise ValueError("lbm3d: mask dimensions must be positive with at most "
                         "geom::max_grid_cells nodes")
    return SolidMask3D(nx, ny, nz, np.zeros(nx * ny * nz, np.uint8), None)


def mask_from_sdf_3d(nx: int, ny: int, nz: int, sdf) -> SolidMask3D:
    """mask_from_sdf_3d (solid_mask3d.cpp:57-75); ``sdf(x, y, z)`` is vectorised."""
    x, y, z = _grid3(nx, ny, nz)
    d = np.asarray(sdf(x, y, z), dtype=np.float64).reshape(-1)
    return SolidMask3D(nx, ny, nz, (d <= 0.0).astype(np.uint8), d)


def sphere_mask(nx: int, ny: int, nz: int, centre, radius: float) -> SolidMask3D:
    """sphere_mask (solid_mask3d.cpp:77-85)."""
    cx, cy, cz = (float(c) for c in centre)

    def sdf(x, y, z):
        dx = x - cx
        dy = y - cy
        dz = z - cz
        return np.sqrt(dx * dx + dy * dy + dz * dz) - radius

    return mask_from_sdf_3d(nx, ny, nz, sdf)


def box_mask(nx: int, ny: int, nz: int, lo, hi) -> SolidMask3D:
    """box_mask (solid_mask3d.cpp:87-102)."""
    lo = [float(v) for v in lo]
    hi = [float(v) for v in hi]

    def sdf(x, y, z):
        p = (x, y, z)
        outside = np.zeros_like(x)
        inside = np.full_like(x, -np.inf)
        for a in range(3):
            excess = np.abs(p[a] - 0.5 * (lo[a] + hi[a])) - 0.5 * (hi[a] - lo[a])
            m = np.maximum(excess, 0.0)
            outside = outside + m * m
            inside = np.maximum(inside, excess)
        return np.sqrt(outside) + np.minimum(inside, 0.0)

    return mask_from_sdf_3d(nx, ny, nz, sdf)


def ellipsoid_mask(nx: int, ny: int, nz: int, centre, semi_axes, angle_z: float = 0.0) -> SolidMask3D:
    """Prolate ellipsoid with semi-axes (a, b, c) along its body axes, rotated by
    ``angle_z`` radians about z (nose up for flow along +x), centred at ``centre``.

    The distance is the first-order estimate (|p/r| - 1) * min(r): exact at the
    surface along the shortest axis, with the right sign everywhere.
    """
    cx, cy, cz = (float(c) for c in centre)
    a, b, c = (float(s) for s in semi_axes)
    ca, sa = math.cos(angle_z), math.sin(angle_z)

    def sdf(x, y, z):
        dx, dy, dz = x - cx, y - cy, z - cz
        # body coordinates: rotate the point by -angle about z
        bx = ca * dx + sa * dy
        by = -sa * dx + ca * dy
        k = np.sqrt((bx / a) ** 2 + (by / b) ** 2 + (dz / c) ** 2)
        return (k - 1.0) * min(a, b, c)

    return mask_from_sdf_3d(nx, ny, nz, sdf)


def sphere_cone_mask(nx: int, ny: int, nz: int, nose, base_radius: float, half_angle: float,
                     nose_radius: float) -> SolidMask3D:
    """Sphere-cone capsule (a blunted cone, axis along +x, base facing downstream):
    a nose sphere of radius ``nose_radius`` tangent to a cone of half-angle
    ``half_angle`` (radians) that opens to ``base_radius``, closed by a flat base.
    ``nose`` is the stagnation point.  Exact signed distance of the solid of
    revolution built from its 2D profile (nose arc, flank, base disc).
    """
    x0, y0, z0 = (float(v) for v in nose)
    rn, rb, th = float(nose_radius), float(base_radius), float(half_angle)
    st, ct = math.sin(th), math.cos(th)
    xc = x0 + rn                       # nose sphere centre on the axis
    xt = xc - rn * st                  # tangency point with the cone (axial)
    rt = rn * ct                       # tangency radius
    length_flank = (rb - rt) / math.tan(th)
    xb = xt + length_flank             # base plane

    def sdf(x, y, z):
        r = np.sqrt((y - y0) ** 2 + (z - z0) ** 2)
        # 2D profile point (s along axis, r radial); distance to the profile polygon
        s = x
        # flank segment from (xt, rt) to (xb, rb)
        ex, er = xb - xt, rb - rt
        ll = ex * ex + er * er
        t = np.clip(((s - xt) * ex + (r - rt) * er) / ll, 0.0, 1.0)
        d_flank = np.hypot(s - (xt + t * ex), r - (rt + t * er))
        # base disc segment from (xb, 0) to (xb, rb)
        rr = np.clip(r, 0.0, rb)
        d_base = np.hypot(s - xb, r - rr)
        # nose arc: points of the sphere with s <= xt
        d_sph = np.abs(np.hypot(s - xc, r) - rn)
        on_arc = (s - xc) * ct <= -(r) * st + 1e-300  # angle test: forward of the tangency ray
        d_arc = np.where(on_arc, d_sph, np.minimum(np.hypot(s - xt, r - rt), np.hypot(s - x0, r)))
        d = np.minimum(np.minimum(d_flank, d_base), d_arc)
        # inside test: within the nose sphere, or between the tangency and base planes under the flank
        inside_sphere = np.hypot(s - xc, r) <= rn
        flank_r = rt + (s - xt) * (er / ex)
        inside_body = (s >= xt) & (s <= xb) & (r <= flank_r)
        inside = inside_sphere | inside_body
        return np.where(inside, -d, d)

    return mask_from_sdf_3d(nx, ny, nz, sdf)


def naca4_profile(digits: str):
    """Camber m, camber position p and thickness t of a NACA 4-digit designation
    (Naca4::from_designation, src/geom/include/orrery/geom/naca.h:36-37)."""
    if len(digits) != 4 or not digits.isdigit():
        raise ValueError(f"not a NACA 4-digit designation: {digits!r}")
    return int(digits[0]) / 100.0, int(digits[1]) / 10.0, int(digits[2:]) / 100.0


def naca_wing_mask(nx: int, ny: int, nz: int, digits: str, leading_edge, chord: float, span: float,
                   angle_of_attack: float) -> SolidMask3D:
    """Straight rectangular wing of a NACA 4-digit section (thickness formula with
    the closed trailing edge, naca.h:21-29), chord along x, thickness along y,
    span along z centred on ``leading_edge[2]``, pitched nose-up by
    ``angle_of_attack`` radians about the leading edge for flow along +x.
    The thickness is laid off normal to the chord line rather than to the
    camber line (a difference of order t theta^2 for the cambered sections).
    The distance is an estimate (positive outside, negative inside) from the
    local half-thickness; the flags are exact point-in-section tests.  The
    section test depends on (x, y) only and the span test on z only, so both
    are evaluated on their own axes and combined by broadcasting.
    """
    if nx <= 0 or ny <= 0 or nz <= 0 or nx * ny * nz > MAX_GRID_CELLS:
        raise ValueError("lbm3d: mask dimensions must be positive with at most "
                         "geom::max_grid_cells nodes")
    m, p, t = naca4_profile(digits)
    lx, ly, lz = (float(v) for v in leading_edge)
    ca, sa = math.cos(angle_of_attack), math.sin(angle_of_attack)
    y, x = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    dx, dy = x - lx, y - ly
    # section coordinates (unit chord): undo the nose-up rotation
    u = (ca * dx - sa * dy) / chord
    v = (sa * dx + ca * dy) / chord
    uc = np.clip(u, 0.0, 1.0)
    yt = 5.0 * t * (0.2969 * np.sqrt(uc) - 0.1260 * uc - 0.3516 * uc ** 2 + 0.2843 * uc ** 3
                    - 0.1036 * uc ** 4)
    if m > 0.0:
        yc = np.where(uc < p, m / p ** 2 * (2 * p * uc - uc ** 2),
                      m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * uc - uc ** 2))
    else:
        yc = np.zeros_like(uc)
    # chordwise and normal excess in lattice units
    d_norm = (np.abs(v - yc) - yt) * chord
    d_chord = np.maximum(-u, u - 1.0) * chord
    d_section = np.maximum(d_norm, d_chord)                        # (ny, nx)
    d_span = np.abs(np.arange(nz, dtype=np.float64) - lz) - 0.5 * span  # (nz,)
    d = np.maximum(d_section[None, :, :], d_span[:, None, None]).reshape(-1)
    return SolidMask3D(nx, ny, nz, (d <= 0.0).astype(np.uint8), d)


def mask_from_sdf(nx: int, ny: int, sdf) -> SolidMask2D:
    """mask_from_sdf (src/aero/lbm/solid_mask.cpp:26-37)."""
    if nx <= 0 or ny <= 0 or nx * ny > MAX_GRID_CELLS:
        raise ValueError("solid mask: dimensions must be at least 1 and the node count at most "
                         "geom::max_grid_cells")
    y, x = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    d = np.asarray(sdf(x.reshape(-1), y.reshape(-1)), dtype=np.float64)
    return SolidMask2D(nx, ny, (d <= 0.0).astype(np.uint8))


def circle_mask(nx: int, ny: int, cx: float, cy: float, radius: float) -> SolidMask2D:
    """circle_mask (src/aero/lbm/solid_mask.cpp:39-43)."""
    return mask_from_sdf(nx, ny, lambda x, y: np.hypot(x - cx, y - cy) - radius)


def fluid_mask(nx: int, ny: int) -> SolidMask2D:
    """fluid_mask (src/aero/lbm/solid_mask.cpp:14-24)."""
    return mask_from_sdf(nx, ny, lambda x, y: np.ones_like(x))
