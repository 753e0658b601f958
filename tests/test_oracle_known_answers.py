"""The reference's own known-answer tests, run on the C restatement.

These restate the analytic checks of tests/aero/lbm3d/test_lbm3d_flows.cpp
(Poiseuille, duct, Couette, co-moving walls, mass, momentum exchange, uniform
stream, inlet next to a sphere, determinism, wall fractions, Smagorinsky
closure) with the same setups and tolerances, so the oracle the CUDA path is
checked against is itself pinned to the reference's published answers.
"""
import math

import numpy as np
import pytest

from helpers import (closure_probe, couette3d_config, duct_config, duct_velocity, poiseuille3d_config, poiseuille3d_velocity,
                     sphere_channel, uniform_state_error)
from oracle import oracle as O
from orrery_b200 import masks as M
from orrery_b200 import solver as S
from orrery_b200.lbm3d import (Lbm3DConfig, Outlet, Smagorinsky, SolidWall, WallKind, XBoundary, periodic_box,
                               wall)


def profile_error(o, cfg, exact):
    rho, ux, uy, uz = o.macroscopic()
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    x = np.tile(np.arange(nx), ny * nz)
    y = np.tile(np.repeat(np.arange(ny), nx), nz)
    z = np.repeat(np.arange(nz), nx * ny)
    e = np.array([exact(a, b, c) for a, b, c in zip(x, y, z)])
    return math.sqrt(np.sum((ux - e) ** 2) / np.sum(e ** 2))


def test_poiseuille_matches_the_parabola():
    """test_lbm3d_flows.cpp:57-68: below 1e-9 at tau = 1/2 + sqrt(3/16), 2e-3 at 0.8."""
    errs = {}
    for tau in (0.5 + math.sqrt(3.0 / 16.0), 0.8):
        cfg = poiseuille3d_config(4, 24, 4, tau, 1e-6)
        o = O.Restated3D(cfg, M.fluid_mask_3d(4, 24, 4).solid)
        o.step(14000)
        errs[tau] = profile_error(o, cfg, lambda x, y, z: poiseuille3d_velocity(cfg, float(y)))
    assert errs[0.5 + math.sqrt(3.0 / 16.0)] < 1e-9
    assert errs[0.8] < 2e-3


def test_square_duct_matches_the_series():
    """test_lbm3d_flows.cpp:70-81."""
    cfg = duct_config(4, 20, 20, 0.5 + math.sqrt(3.0 / 16.0), 1e-6)
    o = O.Restated3D(cfg, M.fluid_mask_3d(4, 20, 20).solid)
    o.step(8000)
    assert profile_error(o, cfg, lambda x, y, z: duct_velocity(cfg, y, z)) < 1e-3


def test_couette():
    """test_lbm3d_flows.cpp:83-93."""
    cfg = couette3d_config(4, 4, 16, 0.8, 0.02)
    o = O.Restated3D(cfg, M.fluid_mask_3d(4, 4, 16).solid)
    o.step(8000)
    assert profile_error(o, cfg, lambda x, y, z: 0.02 * (z + 0.5) / 16.0) < 1e-9


def test_co_moving_walls_at_any_density():
    """test_lbm3d_flows.cpp:95-112."""
    for rho in (0.7, 1.0, 2.0):
        cfg = periodic_box(4, 8, 8, 0.7)
        u = 0.03
        for side in ("y_low", "y_high", "z_low", "z_high"):
            setattr(cfg, side, wall(WallKind.no_slip, u))
        o = O.Restated3D(cfg, M.fluid_mask_3d(4, 8, 8).solid)
        n = cfg.cells
        o.initialize(np.full(n, rho), np.full(n, u), np.zeros(n), np.zeros(n))
        o.step(300)
        r, ux, uy, uz = o.macroscopic()
        assert uniform_state_error(r, ux, uy, uz, rho, (u, 0.0, 0.0), u) < 1e-12


def test_mass_is_conserved():
    """test_lbm3d_flows.cpp:146-168."""
    cfg = periodic_box(12, 10, 9, 0.62)
    cfg.y_low = wall(WallKind.slip)
    cfg.y_high = wall(WallKind.slip)
    cfg.z_low = wall(WallKind.no_slip, 0.02)
    cfg.z_high = wall(WallKind.no_slip, -0.01)
    cfg.smagorinsky = Smagorinsky(True, 0.15)
    mask = M.sphere_mask(12, 10, 9, (6.0, 4.6, 4.2), 2.4)
    o = O.Restated3D(cfg, mask.solid, mask.distance)
    x = np.tile(np.arange(12.0), 90)
    y = np.tile(np.repeat(np.arange(10.0), 12), 9)
    z = np.repeat(np.arange(9.0), 120)
    a = 2 * math.pi * x / 12.0
    o.initialize(1 + 0.01 * np.sin(a), 0.03 * np.cos(a), 0.01 * np.sin(0.7 * y), 0.01 * np.cos(0.5 * z))
    before = o.mass()
    o.step(1500)
    assert abs(o.mass() - before) / before < 1e-12


def test_momentum_exchange_balances_the_body_force():
    """test_lbm3d_flows.cpp:170-188."""
    cfg = periodic_box(4, 16, 4, 0.9)
    cfg.body_force_x = 2e-6
    mask = M.box_mask(4, 16, 4, (0.0, 0.0, 0.0), (3.0, 0.0, 3.0))
    o = O.Restated3D(cfg, mask.solid, mask.distance)
    o.step(6000)
    f = o.force()
    expected = cfg.body_force_x * (4 * 15 * 4)
    assert f[0] == pytest.approx(expected, rel=1e-6)
    assert abs(f[1]) < 1e-12 and abs(f[2]) < 1e-12


def test_uniform_stream_stays_uniform():
    """test_lbm3d_flows.cpp:190-209."""
    for outlet in (Outlet.convective, Outlet.extrapolation):
        cfg = Lbm3DConfig(nx=16, ny=6, nz=5, tau=0.7, outlet=outlet, y_low=wall(WallKind.slip),
                          y_high=wall(WallKind.slip), z_low=wall(WallKind.periodic), z_high=wall(WallKind.periodic),
                          inlet_ux=0.05)
        o = O.Restated3D(cfg, M.fluid_mask_3d(16, 6, 5).solid)
        o.step(400)
        r, ux, uy, uz = o.macroscopic()
        assert uniform_state_error(r, ux, uy, uz, 1.0, (0.05, 0.0, 0.0), 1.0) < 1e-13


def test_inlet_imposes_its_velocity_next_to_a_sphere():
    """test_lbm3d_flows.cpp:211-230."""
    cfg, mask = sphere_channel(40, 20, 20, 8.0, 2.0, 0.05, 20.0)
    cfg.inlet_uy = 0.004
    cfg.inlet_uz = -0.003
    o = O.Restated3D(cfg, mask.solid, mask.distance)
    o.step(600)
    r, ux, uy, uz = o.macroscopic()
    face = np.arange(20 * 20) * 40
    worst = max(np.max(np.abs(ux[face] - 0.05)), np.max(np.abs(uy[face] - 0.004)), np.max(np.abs(uz[face] + 0.003)))
    assert worst < 1e-13
    assert o.force()[0] > 0.0


def test_deterministic_split():
    """test_lbm3d_flows.cpp:232-240."""
    cfg, mask = sphere_channel(32, 16, 16, 6.0, 2.0, 0.05, 50.0)
    a = O.Restated3D(cfg, mask.solid)
    b = O.Restated3D(cfg, mask.solid)
    a.step(150)
    b.step(100)
    b.step(50)
    assert np.array_equal(a.populations(), b.populations())


def fraction_of(fluid, solid, second_solid):
    """Wall fraction of the link (3,4,4) -> (2,4,4) (test_lbm3d_flows.cpp:242-270),
    through the package's host planning."""
    cfg = periodic_box(8, 8, 8, 0.7)
    cfg.solid_wall = SolidWall.interpolated
    mask = M.fluid_mask_3d(8, 8, 8)
    mask.distance = np.ones(mask.solid.size)
    mask.solid = mask.solid.copy()
    mask.solid[mask.index(2, 4, 4)] = 1
    mask.distance[mask.index(2, 4, 4)] = solid
    mask.distance[mask.index(3, 4, 4)] = fluid
    if second_solid:
        mask.solid[mask.index(4, 4, 4)] = 1
        mask.distance[mask.index(4, 4, 4)] = -1.0
    cell, d, q, _, _ = S.plan3d(cfg, mask)
    o = O.Restated3D(cfg, mask.solid, mask.distance)
    oc, od, oq = o.links()
    assert np.array_equal(cell, oc) and np.array_equal(d, od) and np.array_equal(q, oq)
    for c, di, qq in zip(cell, d, q):
        if c == mask.index(3, 4, 4) and di == 1:
            return qq
    raise AssertionError("no link")


def test_wall_fractions_from_the_signed_distance():
    """test_lbm3d_flows.cpp:273-295, on the package's planning and the oracle."""
    inf = math.inf
    big = np.finfo(np.float64).max
    assert fraction_of(0.25, -0.75, False) == 0.25
    assert fraction_of(0.75, -0.25, False) == 0.75
    assert fraction_of(0.0, -1.0, False) == 0.0
    assert fraction_of(1.0, 0.0, False) == 1.0
    assert fraction_of(np.nextafter(0.0, 1.0), 0.0, False) == 1.0
    assert fraction_of(0.25, -0.75, True) == 0.5
    assert fraction_of(0.0, -1.0, True) == 0.5
    assert fraction_of(inf, -1.0, False) == 0.5
    assert fraction_of(1.0, -inf, False) == 0.5
    assert fraction_of(inf, -inf, False) == 0.5
    assert fraction_of(2.0, 1.0, False) == 0.5
    assert fraction_of(-0.5, -1.0, False) == 0.5
    assert fraction_of(0.0, 0.0, False) == 0.5
    assert fraction_of(big, -big, False) == 0.5
    assert fraction_of(big, -0.5 * big, False) == pytest.approx(2.0 / 3.0, rel=1e-15)


def test_smagorinsky_closure_rate():
    """test_lbm3d_flows.cpp:346-384: tau_eff of one collision equals the closure to 1e-10."""
    tau, gamma, cconst = 0.52, 0.01, 0.4
    for a in range(3):
        for b in range(3):
            if a == b:
                continue
            cfg = periodic_box(8, 8, 8, tau)
            cfg.smagorinsky = Smagorinsky(True, cconst)
            o = O.Restated3D(cfg, M.fluid_mask_3d(8, 8, 8).solid)
            n = cfg.cells
            coords = [np.tile(np.arange(8), 64), np.tile(np.repeat(np.arange(8), 8), 8), np.repeat(np.arange(8), 64)]
            u = [np.zeros(n), np.zeros(n), np.zeros(n)]
            u[a] = gamma * (coords[b] - 3.5)
            o.initialize(np.ones(n), *u)
            before = o.populations().reshape(19, n)
            o.step(1)
            after = o.populations().reshape(19, n)
            for k in (1, 3, 6):
                node = [2, 5, 4]
                node[b] = k
                measured, predicted = closure_probe(before, after, node, a, b, tau, cconst)
                assert measured == pytest.approx(predicted, rel=1e-10)
