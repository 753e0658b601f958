"""D3Q19 configuration types mirroring the reference's ``Lbm3DConfig``.

Field names, defaults and meanings follow
``src/aero/lbm3d/include/orrery/aero/lbm3d/lbm3d.h:61-103`` and
``src/aero/lbm/include/orrery/aero/lbm/lbm2d.h:43-78``.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field

from . import abi


class XBoundary(enum.IntEnum):
    """XBoundary (lbm2d.h:43)."""
    periodic = abi.ORR_X_PERIODIC
    inflow_outflow = abi.ORR_X_INFLOW_OUTFLOW


class Outlet(enum.IntEnum):
    """Outlet (lbm2d.h:50)."""
    convective = abi.ORR_OUTLET_CONVECTIVE
    extrapolation = abi.ORR_OUTLET_EXTRAPOLATION


class WallKind(enum.IntEnum):
    """WallKind (lbm2d.h:51)."""
    periodic = abi.ORR_WALL_PERIODIC
    slip = abi.ORR_WALL_SLIP
    no_slip = abi.ORR_WALL_NO_SLIP


class SolidWall(enum.IntEnum):
    """SolidWall (lbm3d.h:81)."""
    halfway = abi.ORR_SOLID_HALFWAY
    interpolated = abi.ORR_SOLID_INTERPOLATED


@dataclass
class Wall:
    """Wall (lbm2d.h:53-56)."""
    kind: WallKind = WallKind.slip
    velocity_x: float = 0.0


@dataclass
class Smagorinsky:
    """Smagorinsky (lbm2d.h:60-63)."""
    enabled: bool = False
    constant: float = 0.1


@dataclass
class Sponge:
    """Sponge (lbm3d.h:61-66)."""
    strength: float = 0.0
    inlet: int = 0
    outlet: int = 0
    sides: int = 0


@dataclass
class Lbm3DConfig:
    """Lbm3DConfig (lbm3d.h:83-103)."""
    nx: int = 0
    ny: int = 0
    nz: int = 0
    tau: float = 0.6
    x_boundary: XBoundary = XBoundary.inflow_outflow
    outlet: Outlet = Outlet.convective
    y_low: Wall = field(default_factory=Wall)
    y_high: Wall = field(default_factory=Wall)
    z_low: Wall = field(default_factory=Wall)
    z_high: Wall = field(default_factory=Wall)
    inlet_ux: float = 0.0
    inlet_uy: float = 0.0
    inlet_uz: float = 0.0
    body_force_x: float = 0.0
    body_force_y: float = 0.0
    body_force_z: float = 0.0
    smagorinsky: Smagorinsky = field(default_factory=Smagorinsky)
    sponge: Sponge = field(default_factory=Sponge)
    solid_wall: SolidWall = SolidWall.halfway

    @property
    def cells(self) -> int:
        return int(self.nx) * int(self.ny) * int(self.nz)

    @classmethod
    def from_c(cls, c: abi.CLbm3DConfig) -> "Lbm3DConfig":
        """The configuration of a C ABI record (the inverse of to_c)."""
        walls = {name: Wall(WallKind(getattr(c, name).kind), getattr(c, name).velocity_x)
                 for name in ("y_low", "y_high", "z_low", "z_high")}
        return cls(nx=c.nx, ny=c.ny, nz=c.nz, tau=c.tau, x_boundary=XBoundary(c.x_boundary),
                   outlet=Outlet(c.outlet), inlet_ux=c.inlet_ux, inlet_uy=c.inlet_uy, inlet_uz=c.inlet_uz,
                   body_force_x=c.body_force_x, body_force_y=c.body_force_y, body_force_z=c.body_force_z,
                   smagorinsky=Smagorinsky(bool(c.smagorinsky_enabled), c.smagorinsky_constant),
                   sponge=Sponge(c.sponge_strength, c.sponge_inlet, c.sponge_outlet, c.sponge_sides),
                   solid_wall=SolidWall(c.solid_wall), **walls)

    def to_c(self) -> abi.CLbm3DConfig:
        c = abi.CLbm3DConfig()
        c.nx, c.ny, c.nz = int(self.nx), int(self.ny), int(self.nz)
        c.tau = float(self.tau)
        c.x_boundary = int(self.x_boundary)
        c.outlet = int(self.outlet)
        for name in ("y_low", "y_high", "z_low", "z_high"):
            w = getattr(self, name)
            cw = getattr(c, name)
            cw.kind = int(w.kind)
            cw.velocity_x = float(w.velocity_x)
        c.inlet_ux, c.inlet_uy, c.inlet_uz = float(self.inlet_ux), float(self.inlet_uy), float(self.inlet_uz)
        c.body_force_x = float(self.body_force_x)
        c.body_force_y = float(self.body_force_y)
        c.body_force_z = float(self.body_force_z)
        c.smagorinsky_enabled = 1 if self.smagorinsky.enabled else 0
        c.smagorinsky_constant = float(self.smagorinsky.constant)
        c.sponge_strength = float(self.sponge.strength)
        c.sponge_inlet = int(self.sponge.inlet)
        c.sponge_outlet = int(self.sponge.outlet)
        c.sponge_sides = int(self.sponge.sides)
        c.solid_wall = int(self.solid_wall)
        return c


@dataclass
class Lbm2DConfig:
    """Lbm2DConfig (lbm2d.h:65-78)."""
    nx: int = 0
    ny: int = 0
    tau: float = 0.6
    x_boundary: XBoundary = XBoundary.inflow_outflow
    outlet: Outlet = Outlet.convective
    bottom: Wall = field(default_factory=Wall)
    top: Wall = field(default_factory=Wall)
    inlet_ux: float = 0.0
    inlet_uy: float = 0.0
    body_force_x: float = 0.0
    body_force_y: float = 0.0
    smagorinsky: Smagorinsky = field(default_factory=Smagorinsky)

    @property
    def cells(self) -> int:
        return int(self.nx) * int(self.ny)

    def to_c(self) -> abi.CLbm2DConfig:
        c = abi.CLbm2DConfig()
        c.nx, c.ny = int(self.nx), int(self.ny)
        c.tau = float(self.tau)
        c.x_boundary = int(self.x_boundary)
        c.outlet = int(self.outlet)
        for name in ("bottom", "top"):
            w = getattr(self, name)
            cw = getattr(c, name)
            cw.kind = int(w.kind)
            cw.velocity_x = float(w.velocity_x)
        c.inlet_ux, c.inlet_uy = float(self.inlet_ux), float(self.inlet_uy)
        c.body_force_x, c.body_force_y = float(self.body_force_x), float(self.body_force_y)
        c.smagorinsky_enabled = 1 if self.smagorinsky.enabled else 0
        c.smagorinsky_constant = float(self.smagorinsky.constant)
        return c


def viscosity_of_tau(tau: float) -> float:
    """viscosity_of_tau (lbm2d.h:89-91): (tau - 1/2) / 3."""
    return (tau - 0.5) / 3.0


def tau_of_viscosity(nu: float) -> float:
    """tau_of_viscosity (lbm2d.h:92-94): 3 nu + 1/2."""
    return nu * 3.0 + 0.5


def wall(kind: WallKind, velocity: float = 0.0) -> Wall:
    return Wall(kind, velocity)


def periodic_box(nx: int, ny: int, nz: int, tau: float) -> Lbm3DConfig:
    """Fully periodic box (tests/aero/lbm3d/lbm3d_test_support.h:66-79)."""
    return Lbm3DConfig(nx=nx, ny=ny, nz=nz, tau=tau, x_boundary=XBoundary.periodic,
                       y_low=wall(WallKind.periodic), y_high=wall(WallKind.periodic),
                       z_low=wall(WallKind.periodic), z_high=wall(WallKind.periodic))
