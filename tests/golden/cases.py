"""Inputs of the golden fixtures: small seeded lattices covering every
boundary option of the path, the validation refusals and the mask builders.
Shared by make_golden.py (which runs the reference on them) and the tests
(which run the restatement and the CUDA path on the same inputs)."""
from __future__ import annotations

import copy

import numpy as np

from orrery_b200 import masks as M
from orrery_b200 import workloads as W
from orrery_b200.lbm3d import (Lbm2DConfig, Lbm3DConfig, Outlet, Smagorinsky, SolidWall, Sponge, WallKind,
                               XBoundary, periodic_box, tau_of_viscosity, wall)


def _sphere_channel(nx=16, ny=10, nz=8, d=4.0, upstream=1.25, u=0.05, re=20.0):
    cfg = Lbm3DConfig(nx=nx, ny=ny, nz=nz, tau=tau_of_viscosity(u * d / re), x_boundary=XBoundary.inflow_outflow,
                      y_low=wall(WallKind.slip), y_high=wall(WallKind.slip), z_low=wall(WallKind.slip),
                      z_high=wall(WallKind.slip), inlet_ux=u)
    mask = M.sphere_mask(nx, ny, nz, (upstream * d, 0.5 * (ny - 1) + 0.25, 0.5 * (nz - 1) + 0.25), 0.5 * d)
    return cfg, mask


def lattice3d_cases():
    """(name, steps, (config, mask, initial fields or None, inlet velocity or None))."""
    out = []
    cfg, mask = _sphere_channel()
    init = W.noisy_state3d(cfg, mask, seed=11)
    out.append(("sphere_bgk", 60, (cfg, mask, init, None)))
    les = copy.deepcopy(cfg)
    les.smagorinsky = Smagorinsky(True, 0.1)
    les.outlet = Outlet.extrapolation
    out.append(("sphere_les_extrapolation", 60, (les, mask, init, None)))
    interp = copy.deepcopy(cfg)
    interp.solid_wall = SolidWall.interpolated
    out.append(("sphere_interpolated", 60, (interp, mask, init, None)))
    sponge = copy.deepcopy(cfg)
    sponge.sponge = Sponge(0.5, 3, 4, 2)
    out.append(("sphere_sponge_ramped_inlet", 60, (sponge, mask, init, (0.03, 0.002, -0.001))))
    sides = copy.deepcopy(cfg)
    sides.y_low = wall(WallKind.periodic)
    sides.y_high = wall(WallKind.periodic)
    sides.z_low = wall(WallKind.no_slip, 0.01)
    sides.z_high = wall(WallKind.no_slip, -0.015)
    sides.inlet_uy = 0.004
    out.append(("sphere_periodic_y_moving_z", 60, (sides, mask, init, None)))
    box = periodic_box(12, 10, 9, 0.62)
    box.y_low = wall(WallKind.slip)
    box.y_high = wall(WallKind.slip)
    box.z_low = wall(WallKind.no_slip, 0.02)
    box.z_high = wall(WallKind.no_slip, -0.01)
    box.smagorinsky = Smagorinsky(True, 0.15)
    box.body_force_x = 1e-5
    box.body_force_z = -2e-6
    bmask = M.sphere_mask(12, 10, 9, (6.0, 4.6, 4.2), 2.4)
    n = box.cells
    rho = 1.0 + W.uniform_noise(5, n, 3, 0.01)
    ux = 0.03 + W.uniform_noise(5, n, 0, 0.01)
    uy = W.uniform_noise(5, n, 1, 0.01)
    uz = W.uniform_noise(5, n, 2, 0.01)
    out.append(("periodic_box_forced_walls", 120, (box, bmask, (rho, ux, uy, uz), None)))
    return out


def lattice2d_cases():
    """(name, steps, (config, mask, initial fields or None))."""
    out = []
    cfg = Lbm2DConfig(nx=40, ny=20, tau=tau_of_viscosity(0.05 * 8 / 40.0), x_boundary=XBoundary.inflow_outflow,
                      outlet=Outlet.extrapolation, bottom=wall(WallKind.slip), top=wall(WallKind.slip),
                      inlet_ux=0.05, smagorinsky=Smagorinsky(True, 0.1))
    mask = M.circle_mask(40, 20, 12.0, 9.6, 4.0)
    n = cfg.cells
    fluid = mask.solid == 0
    init = (np.ones(n), np.where(fluid, 0.05 + W.uniform_noise(13, n, 0, 1e-3), 0.0),
            np.where(fluid, W.uniform_noise(13, n, 1, 1e-3), 0.0))
    out.append(("cylinder_les_extrapolation", 100, (cfg, mask, init)))
    conv = copy.deepcopy(cfg)
    conv.outlet = Outlet.convective
    conv.inlet_uy = 0.004
    conv.smagorinsky = Smagorinsky(False, 0.1)
    out.append(("cylinder_convective_skewed", 100, (conv, mask, init)))
    walls = Lbm2DConfig(nx=24, ny=16, tau=0.7, x_boundary=XBoundary.periodic, bottom=wall(WallKind.no_slip, 0.01),
                        top=wall(WallKind.no_slip, -0.02), body_force_x=1e-5, body_force_y=2e-6)
    wmask = M.circle_mask(24, 16, 10.0, 8.0, 3.0)
    m = walls.cells
    winit = (1.0 + W.uniform_noise(17, m, 2, 0.01), W.uniform_noise(17, m, 0, 0.02), W.uniform_noise(17, m, 1, 0.01))
    out.append(("periodic_moving_walls_forced", 200, (walls, wmask, winit)))
    return out


def sphere_masks():
    return {"sphere_off_grid": (17, 9, 11, (8.3, 4.1, 5.7), 3.3), "sphere_on_grid": (12, 12, 12, (6.0, 6.0, 6.0), 4.0)}


def box_masks():
    return {"box_plate": (10, 8, 6, (2.0, 3.0, 1.0), (6.5, 3.0, 4.0))}


def circle_masks():
    return {"circle_off_grid": (31, 17, 12.4, 8.3, 5.1)}


def validation_cases3d():
    """(label, config, mask) covering each refusal of validate()."""
    out = []
    fm = M.fluid_mask_3d(8, 8, 8)
    ok = periodic_box(8, 8, 8, 0.6)
    out.append(("accepted", ok, fm))
    c = copy.deepcopy(ok); c.tau = 0.5
    out.append(("tau", c, fm))
    c = copy.deepcopy(ok); c.body_force_z = float("inf")
    out.append(("infinite force", c, fm))
    c = copy.deepcopy(ok); c.smagorinsky = Smagorinsky(True, -0.1)
    out.append(("negative Smagorinsky", c, fm))
    c = copy.deepcopy(ok); c.z_low = wall(WallKind.slip)
    out.append(("half periodic", c, fm))
    c = copy.deepcopy(ok); c.y_low = wall(WallKind.no_slip, 0.06); c.y_high = wall(WallKind.no_slip)
    out.append(("fast wall", c, fm))
    ch = copy.deepcopy(ok); ch.x_boundary = XBoundary.inflow_outflow; ch.inlet_ux = 0.05
    out.append(("channel", ch, fm))
    c = copy.deepcopy(ch); c.inlet_uz = 0.04
    out.append(("inlet Mach", c, fm))
    c = copy.deepcopy(ch); c.inlet_ux = 0.08
    out.append(("inlet 0.08", c, fm))
    out.append(("blocked outlet", ch, M.box_mask(8, 8, 8, (7.0, 3.0, 3.0), (7.0, 3.0, 3.0))))
    c = copy.deepcopy(ch); c.inlet_ux = 0.0
    out.append(("convective without inflow", c, fm))
    c = copy.deepcopy(ch); c.inlet_ux = 0.0; c.outlet = Outlet.extrapolation
    out.append(("extrapolation without inflow", c, fm))
    c = copy.deepcopy(ch); c.sponge = Sponge(1.5, 2, 2, 2)
    out.append(("sponge strength", c, fm))
    c = copy.deepcopy(ch); c.sponge = Sponge(0.5, 9, 2, 2)
    out.append(("sponge too thick", c, fm))
    c = copy.deepcopy(ok); c.sponge = Sponge(0.5, 2, 2, 2)
    out.append(("sponge periodic", c, fm))
    c = copy.deepcopy(ch); c.solid_wall = SolidWall.interpolated
    out.append(("interpolated without distance", c, fm))
    nan_mask = M.sphere_mask(8, 8, 8, (4.0, 4.0, 4.0), 1.5)
    nan_mask.distance = nan_mask.distance.copy(); nan_mask.distance[5] = float("nan")
    out.append(("interpolated NaN distance", c, nan_mask))
    c = copy.deepcopy(ok); c.nz = 2
    out.append(("too small", c, M.fluid_mask_3d(8, 8, 2)))
    return out


def validation_cases2d():
    out = []
    fm = M.fluid_mask(8, 8)
    ok = Lbm2DConfig(nx=8, ny=8, tau=0.6, x_boundary=XBoundary.periodic, bottom=wall(WallKind.periodic),
                     top=wall(WallKind.periodic))
    out.append(("accepted", ok, fm))
    c = copy.deepcopy(ok); c.tau = 0.4
    out.append(("tau", c, fm))
    c = copy.deepcopy(ok); c.bottom = wall(WallKind.slip)
    out.append(("half periodic", c, fm))
    c = copy.deepcopy(ok); c.bottom = wall(WallKind.no_slip, 0.07); c.top = wall(WallKind.no_slip)
    out.append(("fast wall", c, fm))
    ch = copy.deepcopy(ok); ch.x_boundary = XBoundary.inflow_outflow; ch.inlet_ux = 0.05
    out.append(("channel", ch, fm))
    c = copy.deepcopy(ch); c.inlet_uy = 0.045
    out.append(("inlet Mach", c, fm))
    c = copy.deepcopy(ch); c.inlet_ux = 0.0
    out.append(("convective without inflow", c, fm))
    blocked = M.fluid_mask(8, 8); blocked.solid = blocked.solid.copy(); blocked.solid[7 + 8 * 3] = 1
    out.append(("blocked outlet", ch, blocked))
    return out
