"""Seeded synthetic workloads of the LBM path and the coefficient arithmetic.

Each builder returns the lattice configuration, its solid mask and the
initial macroscopic fields.  Initial velocities carry seeded uniform noise
of +-1e-3 per component at fluid nodes, drawn from a counter-based generator
(SplitMix64 of seed, node and component), so any host reproduces the same
inputs without shipping them.

Workloads (sizes in lattice nodes):
  cylinder2d      D2Q9 400 x 160, circle D = 32 at (100, 80), u = 0.05,
                  Re 100 (nu 0.016, tau 0.548), Smagorinsky C = 0.1,
                  zero-gradient outflow, free-slip top and bottom.
  sphere3d        D3Q19 256 x 128 x 128, sphere D = 32 at (64, 64, 64),
                  u = 0.05, Re 200 (nu 0.008, tau 0.524), Smagorinsky
                  C = 0.1, zero-gradient outflow, free-slip lateral walls.
  ellipsoid3d     D3Q19 512 x 256 x 256, prolate ellipsoid (48, 24, 24)
                  rotated 10 degrees about z, u = 0.08, Re 1000 on the major
                  axis L = 96 (nu 0.00768), Smagorinsky C = 0.12 (the inlet
                  speed is above the lattice Mach guard: needs the opt-in).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import masks as M
from .lbm3d import (Lbm2DConfig, Lbm3DConfig, Outlet, Smagorinsky, SolidWall, WallKind,
                    XBoundary, tau_of_viscosity, wall)

_MASK64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea and Flood 2014) on uint64 arrays."""
    z = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_MASK64)
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_MASK64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_MASK64)
    return z ^ (z >> np.uint64(31))


def uniform_noise(seed: int, cells: int, component: int, amplitude: float) -> np.ndarray:
    """amplitude * U(-1, 1) per node from SplitMix64(seed * 2^32 + 4 node + component)."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) << np.uint64(32)) + np.arange(cells, dtype=np.uint64) * np.uint64(4) \
            + np.uint64(component)
        bits = splitmix64(key) >> np.uint64(11)  # 53 random bits
    u = bits.astype(np.float64) * (1.0 / 9007199254740992.0)  # [0, 1)
    return amplitude * (2.0 * u - 1.0)


@dataclass
class Workload3D:
    name: str
    config: Lbm3DConfig
    mask: M.SolidMask3D
    rho: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    uz: np.ndarray
    reference_length: float   # D (sphere) or L (ellipsoid)
    reference_area: float     # frontal area of the coefficients
    allow_high_mach: bool = False

    @property
    def cells(self) -> int:
        return self.config.cells


@dataclass
class Workload2D:
    name: str
    config: Lbm2DConfig
    mask: M.SolidMask2D
    rho: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    reference_length: float


def noisy_state3d(config: Lbm3DConfig, mask, seed: int, amplitude: float = 1e-3):
    n = config.cells
    fluid = mask.solid == 0
    rho = np.ones(n)
    ux = np.where(fluid, config.inlet_ux + uniform_noise(seed, n, 0, amplitude), 0.0)
    uy = np.where(fluid, config.inlet_uy + uniform_noise(seed, n, 1, amplitude), 0.0)
    uz = np.where(fluid, config.inlet_uz + uniform_noise(seed, n, 2, amplitude), 0.0)
    return rho, ux, uy, uz


def sphere3d(seed: int = 1, nx: int = 256, ny: int = 128, nz: int = 128, diameter: float = 32.0,
             centre=None, u: float = 0.05, reynolds: float = 200.0, smagorinsky: float = 0.1,
             outlet: Outlet = Outlet.extrapolation, noise: float = 1e-3) -> Workload3D:
    """Sphere in a channel; the defaults are the 256 x 128 x 128, D 32, Re 200 case."""
    centre = centre if centre is not None else (nx / 4.0, ny / 2.0, nz / 2.0)
    cfg = Lbm3DConfig(nx=nx, ny=ny, nz=nz, tau=tau_of_viscosity(u * diameter / reynolds),
                      x_boundary=XBoundary.inflow_outflow, outlet=outlet,
                      y_low=wall(WallKind.slip), y_high=wall(WallKind.slip),
                      z_low=wall(WallKind.slip), z_high=wall(WallKind.slip), inlet_ux=u,
                      smagorinsky=Smagorinsky(smagorinsky > 0.0, smagorinsky))
    mask = M.sphere_mask(nx, ny, nz, centre, 0.5 * diameter)
    rho, ux, uy, uz = noisy_state3d(cfg, mask, seed, noise)
    return Workload3D(f"sphere3d_{nx}x{ny}x{nz}", cfg, mask, rho, ux, uy, uz, diameter,
                      math.pi * diameter * diameter / 4.0)


def ellipsoid3d(seed: int = 1, nx: int = 512, ny: int = 256, nz: int = 256, semi=(48.0, 24.0, 24.0),
                angle_deg: float = 10.0, u: float = 0.08, reynolds: float = 1000.0,
                smagorinsky: float = 0.12, centre=None, noise: float = 1e-3) -> Workload3D:
    """Prolate ellipsoid at an angle of attack; the defaults are the 512 x 256 x 256 case.
    Re is on the major axis L = 2 a; the lift acts along y."""
    scale = nx / 512.0
    semi = tuple(s * scale for s in semi)
    centre = centre if centre is not None else (nx / 4.0, ny / 2.0, nz / 2.0)
    length = 2.0 * semi[0]
    cfg = Lbm3DConfig(nx=nx, ny=ny, nz=nz, tau=tau_of_viscosity(u * length / reynolds),
                      x_boundary=XBoundary.inflow_outflow, outlet=Outlet.extrapolation,
                      y_low=wall(WallKind.slip), y_high=wall(WallKind.slip),
                      z_low=wall(WallKind.slip), z_high=wall(WallKind.slip), inlet_ux=u,
                      smagorinsky=Smagorinsky(True, smagorinsky))
    mask = M.ellipsoid_mask(nx, ny, nz, centre, semi, math.radians(angle_deg))
    rho, ux, uy, uz = noisy_state3d(cfg, mask, seed, noise)
    return Workload3D(f"ellipsoid3d_{nx}x{ny}x{nz}", cfg, mask, rho, ux, uy, uz, length,
                      math.pi * semi[1] * semi[2], allow_high_mach=True)


def cylinder2d(seed: int = 1, nx: int = 400, ny: int = 160, diameter: float = 32.0, centre=(100.0, 80.0),
               u: float = 0.05, reynolds: float = 100.0, smagorinsky: float = 0.1,
               noise: float = 1e-3) -> Workload2D:
    """Cylinder in a channel; the defaults are the 400 x 160, D 32, Re 100 case."""
    cfg = Lbm2DConfig(nx=nx, ny=ny, tau=tau_of_viscosity(u * diameter / reynolds),
                      x_boundary=XBoundary.inflow_outflow, outlet=Outlet.extrapolation,
                      bottom=wall(WallKind.slip), top=wall(WallKind.slip), inlet_ux=u,
                      smagorinsky=Smagorinsky(smagorinsky > 0.0, smagorinsky))
    mask = M.circle_mask(nx, ny, centre[0], centre[1], 0.5 * diameter)
    n = cfg.cells
    fluid = mask.solid == 0
    rho = np.ones(n)
    ux = np.where(fluid, u + uniform_noise(seed, n, 0, noise), 0.0)
    uy = np.where(fluid, uniform_noise(seed, n, 1, noise), 0.0)
    return Workload2D(f"cylinder2d_{nx}x{ny}", cfg, mask, rho, ux, uy, diameter)


def coefficients3d(force, moment, u: float, area: float, length: float, rho: float = 1.0,
                   centre=(0.0, 0.0, 0.0)):
    """Cd, Cl (lift along +y), Cy (side force along z) and Cm (pitching moment
    about z through ``centre``): F / (1/2 rho U^2 A), M / (1/2 rho U^2 A L)
    (set_coefficients, src/aero/include/orrery/aero/aero_result.h:92;
    the moment shift of lbm_aero_solver3d.cpp:428-431)."""
    q = 0.5 * rho * u * u
    f = np.asarray(force, dtype=np.float64)
    m = np.asarray(moment, dtype=np.float64)
    c = np.asarray(centre, dtype=np.float64)
    m_c = m - np.cross(c, f)  # moment about the centre
    return {"cd": f[0] / (q * area), "cl": f[1] / (q * area), "cy": f[2] / (q * area),
            "cm": m_c[2] / (q * area * length)}


def coefficients2d(fx: float, fy: float, u: float, diameter: float, rho: float = 1.0):
    """force_coefficients (src/aero/lbm/force_history.cpp:9-13): per unit span."""
    q = 0.5 * rho * u * u
    return {"cd": fx / (q * diameter), "cl": fy / (q * diameter)}
