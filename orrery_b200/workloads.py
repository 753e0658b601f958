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
  naca_batch      64 D3Q19 lattices for the batched form: sizes drawn from the
                  seed between 96^3 and 256 x 128 x 128 (nx a multiple of 16),
                  each with a NACA 4-digit wing (0012, 2412 or 4415), chord
                  0.4 nx, span 0.6 nz, angle of attack uniform in -4..12
                  degrees, u = 0.05, Re uniform in 200..1000 on the chord,
                  Smagorinsky C = 0.1, free-slip lateral walls, zero-gradient
                  outflow.
  reference_benchmarks
                  the reference's own GPU benchmark cases
                  (tests/bench/aero/bench_lbm_gpu.cpp:91-140): the D3Q19 128^3
                  sphere channel (D 24 a quarter node off the axis, 2.5 D from
                  the inlet, u = 0.05, Re 300, free-slip sides) and the D2Q9
                  2048 x 1024 cylinder (D 64 at (400, 512.5), u = 0.05,
                  Re 1000, free-slip top and bottom), each without and with
                  the Smagorinsky closure (C = 0.1), from the uniform inlet
                  state.
  sphere_cone_requests
                  the serving form's request stream: Poisson arrivals (rate
                  20/s), sphere-cone capsules (half-angle 20..35 degrees, nose
                  radius 0.2..0.4 of the base radius, base radius ny / 8) on
                  grids nx = 64 + 256 t, ny = nz = 64 + 96 t with t uniform in
                  [0, 1] (nx rounded to a multiple of 16), Re uniform in
                  100..2000 on the base diameter, u = 0.05, Smagorinsky C = 0.1.
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


@dataclass
class BenchmarkCase:
    """One of the reference's GPU benchmark cases and its published rate on
    its OpenGL backend (AMD Radeon RX 9060 XT, binary32;
    docs/performance.md:140-141, 164)."""
    name: str
    config: object
    mask: object
    cells: int
    published_steps_per_s: float


def reference_benchmarks() -> list[BenchmarkCase]:
    """The four cases of tests/bench/aero/bench_lbm_gpu.cpp (sphere_channel,
    lbm3d_test_support.h:249-270; cylinder_setup, lbm_test_support.h:
    154-167)."""
    cases = []
    published = {(3, False): 681.86, (3, True): 676.67, (2, False): 1521.0, (2, True): 1475.0}
    for les in (False, True):
        n, d, u = 128, 24.0, 0.05
        c = Lbm3DConfig(nx=n, ny=n, nz=n, tau=tau_of_viscosity(u * d / 300.0),
                        x_boundary=XBoundary.inflow_outflow, y_low=wall(WallKind.slip),
                        y_high=wall(WallKind.slip), z_low=wall(WallKind.slip), z_high=wall(WallKind.slip),
                        inlet_ux=u, smagorinsky=Smagorinsky(les, 0.1))
        centre = (2.5 * d, 0.5 * (n - 1) + 0.25, 0.5 * (n - 1) + 0.25)
        cases.append(BenchmarkCase(f"sphere3d_128^3_{'les' if les else 'bgk'}", c,
                                   M.sphere_mask(n, n, n, centre, 0.5 * d), n ** 3, published[(3, les)]))
    for les in (False, True):
        nx, ny, d, u = 2048, 1024, 64.0, 0.05
        c = Lbm2DConfig(nx=nx, ny=ny, tau=tau_of_viscosity(u * d / 1000.0),
                        x_boundary=XBoundary.inflow_outflow, bottom=wall(WallKind.slip),
                        top=wall(WallKind.slip), inlet_ux=u, smagorinsky=Smagorinsky(les, 0.1))
        cases.append(BenchmarkCase(f"cylinder2d_2048x1024_{'les' if les else 'bgk'}", c,
                                   M.circle_mask(nx, ny, 400.0, 512.5, 0.5 * d), nx * ny, published[(2, les)]))
    return cases


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


@dataclass
class BatchMember:
    """Parameters of one lattice of the batched form; ``build()`` makes the workload."""
    index: int
    seed: int
    nx: int
    ny: int
    nz: int
    digits: str
    angle_deg: float
    reynolds: float
    u: float = 0.05
    smagorinsky: float = 0.1
    noise: float = 1e-3

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def chord(self) -> float:
        return 0.4 * self.nx

    @property
    def span(self) -> float:
        return 0.6 * self.nz

    def build(self) -> Workload3D:
        chord = self.chord
        cfg = Lbm3DConfig(nx=self.nx, ny=self.ny, nz=self.nz,
                          tau=tau_of_viscosity(self.u * chord / self.reynolds),
                          x_boundary=XBoundary.inflow_outflow, outlet=Outlet.extrapolation,
                          y_low=wall(WallKind.slip), y_high=wall(WallKind.slip),
                          z_low=wall(WallKind.slip), z_high=wall(WallKind.slip), inlet_ux=self.u,
                          smagorinsky=Smagorinsky(self.smagorinsky > 0.0, self.smagorinsky))
        leading = (0.25 * self.nx, 0.5 * self.ny, 0.5 * self.nz)
        mask = M.naca_wing_mask(self.nx, self.ny, self.nz, self.digits, leading, chord, self.span,
                                math.radians(self.angle_deg))
        rho, ux, uy, uz = noisy_state3d(cfg, mask, self.seed, self.noise)
        return Workload3D(f"naca{self.digits}_{self.nx}x{self.ny}x{self.nz}", cfg, mask, rho, ux, uy, uz,
                          chord, chord * self.span)


def naca_batch(seed: int = 4, count: int = 64) -> list[BatchMember]:
    """The batched form's lattices (see the module docstring)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nx = int(16 * round(rng.uniform(96.0, 256.0) / 16.0))
        ny = int(round(rng.uniform(96.0, 128.0)))
        nz = int(round(rng.uniform(96.0, 128.0)))
        digits = str(rng.choice(["0012", "2412", "4415"]))
        angle = float(rng.uniform(-4.0, 12.0))
        reynolds = float(rng.uniform(200.0, 1000.0))
        out.append(BatchMember(k, seed * 1000 + k, nx, ny, nz, digits, angle, reynolds))
    return out


@dataclass
class SolveRequest:
    """One request of the serving form: arrival time (seconds from the
    start of the stream) and the body; ``build()`` makes the workload."""
    index: int
    seed: int
    arrival: float
    nx: int
    ny: int
    nz: int
    half_angle_deg: float
    nose_ratio: float
    reynolds: float
    u: float = 0.05
    smagorinsky: float = 0.1
    noise: float = 1e-3

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def base_radius(self) -> float:
        return self.ny / 8.0

    def build(self) -> Workload3D:
        rb = self.base_radius
        diameter = 2.0 * rb
        cfg = Lbm3DConfig(nx=self.nx, ny=self.ny, nz=self.nz,
                          tau=tau_of_viscosity(self.u * diameter / self.reynolds),
                          x_boundary=XBoundary.inflow_outflow, outlet=Outlet.extrapolation,
                          y_low=wall(WallKind.slip), y_high=wall(WallKind.slip),
                          z_low=wall(WallKind.slip), z_high=wall(WallKind.slip), inlet_ux=self.u,
                          smagorinsky=Smagorinsky(self.smagorinsky > 0.0, self.smagorinsky))
        nose = (0.2 * self.nx, 0.5 * (self.ny - 1), 0.5 * (self.nz - 1))
        mask = M.sphere_cone_mask(self.nx, self.ny, self.nz, nose, rb, math.radians(self.half_angle_deg),
                                  self.nose_ratio * rb)
        rho, ux, uy, uz = noisy_state3d(cfg, mask, self.seed, self.noise)
        return Workload3D(f"sphere_cone_{self.nx}x{self.ny}x{self.nz}", cfg, mask, rho, ux, uy, uz,
                          diameter, math.pi * rb * rb)


def sphere_cone_requests(seed: int = 5, count: int = 48, rate: float = 20.0) -> list[SolveRequest]:
    """The serving form's request stream (see the module docstring)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += float(rng.exponential(1.0 / rate))
        size = float(rng.uniform(0.0, 1.0))
        nx = int(16 * round((64.0 + 256.0 * size) / 16.0))
        ny = nz = int(round(64.0 + 96.0 * size))
        out.append(SolveRequest(k, seed * 1000 + k, t, nx, ny, nz, float(rng.uniform(20.0, 35.0)),
                                float(rng.uniform(0.2, 0.4)), float(rng.uniform(100.0, 2000.0))))
    return out
