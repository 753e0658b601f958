"""D2Q9 CUDA path against the CPU oracle on identical inputs.

The 400 x 160 cylinder channel (D 32 at (100, 80), u 0.05, Re 100,
Smagorinsky C 0.1, zero-gradient outflow, free-slip walls, seeded +-1e-3
noise) and the reference's analytic 2D flows
(tests/aero/lbm/test_lbm_gpu.cpp, test_lbm2d_flows.cpp).
"""
import math

import numpy as np
import pytest

from helpers import copy_config, l2_relative, velocity_l2
from oracle import oracle as O
from orrery_b200 import masks as M
from orrery_b200 import solver as S
from orrery_b200 import workloads as W
from orrery_b200.lbm3d import (Lbm2DConfig, Outlet, WallKind, XBoundary, viscosity_of_tau, wall)

pytestmark = pytest.mark.gpu


def run_both(config, mask, steps, storage="f32", init=None):
    g = S.make_gpu_solver(config, mask, storage=storage)
    o = O.Restated2D(config, mask.solid)
    if init is not None:
        g.initialize(*init)
        o.initialize(*init)
    g.step(steps)
    o.step(steps)
    return g, o


def test_cylinder_binary32_1000_steps():
    w = W.cylinder2d(seed=3)
    g, o = run_both(w.config, w.mask, 1000, init=(w.rho, w.ux, w.uy))
    pops = l2_relative(g.populations(), o.populations())
    mg = g.macroscopic()
    _, uxo, uyo = o.macroscopic()
    vel = velocity_l2([mg.velocity_x, mg.velocity_y], [uxo, uyo], w.mask.solid)
    fg, fo = g.force(), o.force()
    cd_g = W.coefficients2d(fg.x, fg.y, 0.05, 32.0)["cd"]
    cd_o = W.coefficients2d(fo[0], fo[1], 0.05, 32.0)["cd"]
    print(f"measured: D2Q9 f32 vs CPU cylinder 1000 steps: populations L2 {pops:.3e}, velocity L2 {vel:.3e}, "
          f"Cd {cd_g:.6f} vs {cd_o:.6f}")
    assert pops < 1e-5
    assert abs(cd_g - cd_o) / abs(cd_o) < 1e-4


def test_cylinder_binary64_is_bitwise():
    w = W.cylinder2d(seed=3)
    g, o = run_both(w.config, w.mask, 300, storage="f64", init=(w.rho, w.ux, w.uy))
    assert np.array_equal(g.populations(), o.populations())
    mg = g.macroscopic()
    mo = o.macroscopic()
    assert np.array_equal(mg.density, mo[0])
    assert np.array_equal(mg.velocity_x, mo[1])
    assert np.array_equal(mg.velocity_y, mo[2])
    fg, fo = g.force(), o.force()
    assert abs(fg.x - fo[0]) < 1e-12 and abs(fg.y - fo[1]) < 1e-12 and abs(fg.moment - fo[2]) < 1e-10


def test_walls_force_convective_binary64_bitwise():
    cfg = Lbm2DConfig(nx=64, ny=40, tau=0.62, x_boundary=XBoundary.inflow_outflow, outlet=Outlet.convective,
                      bottom=wall(WallKind.no_slip, 0.01), top=wall(WallKind.slip), inlet_ux=0.04,
                      inlet_uy=0.005, body_force_x=1e-6, body_force_y=-3e-7)
    cfg.smagorinsky.enabled = True
    mask = M.circle_mask(64, 40, 20.0, 19.5, 5.0)
    g, o = run_both(cfg, mask, 400, storage="f64")
    assert np.array_equal(g.populations(), o.populations())


def test_periodic_walls_binary32():
    cfg = Lbm2DConfig(nx=48, ny=32, tau=0.7, x_boundary=XBoundary.periodic,
                      bottom=wall(WallKind.periodic), top=wall(WallKind.periodic), body_force_x=2e-6)
    mask = M.circle_mask(48, 32, 24.0, 16.0, 4.0)
    g, o = run_both(cfg, mask, 2000)
    assert l2_relative(g.populations(), o.populations()) < 1e-5


def test_poiseuille_2d_against_cpu():
    tau = 0.8
    cfg = Lbm2DConfig(nx=4, ny=32, tau=tau, x_boundary=XBoundary.periodic,
                      bottom=wall(WallKind.no_slip), top=wall(WallKind.no_slip), body_force_x=1e-6)
    mask = M.fluid_mask(4, 32)
    g, o = run_both(cfg, mask, 4000)
    mg = g.macroscopic()
    _, uxo, uyo = o.macroscopic()
    vel = velocity_l2([mg.velocity_x, mg.velocity_y], [uxo, uyo], mask.solid)
    nu = viscosity_of_tau(tau)
    y = np.repeat(np.arange(32.0), 4)
    exact = 1e-6 / (2 * nu) * (y + 0.5) * (32 - 0.5 - y)
    err = math.sqrt(np.sum((mg.velocity_x - exact) ** 2) / np.sum(exact ** 2))
    print(f"measured: D2Q9 f32 Poiseuille vs CPU {vel:.3e}, vs parabola {err:.3e}")
    assert vel < 1e-4
    assert err < 5e-2


def test_links_match_the_oracle_2d():
    w = W.cylinder2d(seed=3)
    g = S.make_gpu_solver(w.config, w.mask)
    o = O.Restated2D(w.config, w.mask.solid)
    for a, b in zip(g.links(), o.links()):
        assert np.array_equal(a, b)
