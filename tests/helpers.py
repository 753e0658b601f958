"""Shared helpers of the tests: the configurations and error norms of the
reference's test support headers (tests/aero/lbm/lbm_test_support.h,
tests/aero/lbm3d/lbm3d_test_support.h), restated for numpy."""
from __future__ import annotations

import math

import numpy as np

from orrery_b200 import masks as M
from orrery_b200.lbm3d import (Lbm2DConfig, Lbm3DConfig, Outlet, Smagorinsky, WallKind, XBoundary,
                               periodic_box, tau_of_viscosity, viscosity_of_tau, wall)


def l2_relative(a, b, skip=None):
    """||a - b|| / ||b|| over entries where skip is 0 (lbm_test_support.h:34-47)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if skip is not None:
        keep = np.asarray(skip) == 0
        a, b = a[keep], b[keep]
    diff = float(np.sum((a - b) ** 2))
    norm = float(np.sum(b * b))
    return math.sqrt(diff / norm) if norm > 0 else math.sqrt(diff)


def velocity_l2(a_fields, b_fields, solid):
    """Relative L2 of the velocity over fluid nodes (lbm3d_test_support.h:23-35)."""
    va = np.concatenate([np.asarray(v) for v in a_fields])
    vb = np.concatenate([np.asarray(v) for v in b_fields])
    skip = np.concatenate([solid] * len(a_fields))
    return l2_relative(va, vb, skip)


def uniform_state_error(rho, ux, uy, uz, rho0, u, scale):
    """Largest deviation from a uniform state; inf for non-finite values
    (lbm3d_test_support.h:47-60)."""
    parts = [np.abs(np.asarray(rho) - rho0) / rho0, np.abs(np.asarray(ux) - u[0]) / scale,
             np.abs(np.asarray(uy) - u[1]) / scale, np.abs(np.asarray(uz) - u[2]) / scale]
    worst = 0.0
    for p in parts:
        if not np.all(np.isfinite(p)):
            return math.inf
        worst = max(worst, float(np.max(p)))
    return worst


def poiseuille3d_config(nx, ny, nz, tau, g):
    c = periodic_box(nx, ny, nz, tau)
    c.y_low = wall(WallKind.no_slip)
    c.y_high = wall(WallKind.no_slip)
    c.body_force_x = g
    return c


def poiseuille3d_velocity(config, y):
    nu = viscosity_of_tau(config.tau)
    h = float(config.ny)
    return config.body_force_x / (2.0 * nu) * (y + 0.5) * (h - 0.5 - y)


def duct_config(nx, ny, nz, tau, g):
    c = poiseuille3d_config(nx, ny, nz, tau, g)
    c.z_low = wall(WallKind.no_slip)
    c.z_high = wall(WallKind.no_slip)
    return c


def duct_velocity(config, yi, zi):
    """White, Viscous Fluid Flow, eq. 3-48 series (lbm3d_test_support.h:99-131)."""
    nu = viscosity_of_tau(config.tau)
    a = 0.5 * config.ny
    b = 0.5 * config.nz
    y = yi - 0.5 * (config.ny - 1)
    z = zi - 0.5 * (config.nz - 1)
    total = 0.0
    for n in range(1, 200, 2):
        k = n * math.pi / (2.0 * a)
        sign = 1.0 if ((n - 1) // 2) % 2 == 0 else -1.0
        ratio = math.exp(k * (abs(z) - b)) * (1.0 + math.exp(-2.0 * k * abs(z))) / (1.0 + math.exp(-2.0 * k * b))
        total += sign / (n * n * n) * (1.0 - ratio) * math.cos(k * y)
    return 16.0 * a * a * config.body_force_x / (nu * math.pi ** 3) * total


def couette3d_config(nx, ny, nz, tau, u_wall):
    c = periodic_box(nx, ny, nz, tau)
    c.z_low = wall(WallKind.no_slip)
    c.z_high = wall(WallKind.no_slip, u_wall)
    return c


def sphere_channel(nx, ny, nz, diameter, upstream, u, reynolds):
    """Sphere a quarter node off the channel axis (lbm3d_test_support.h:241-270)."""
    c = Lbm3DConfig(nx=nx, ny=ny, nz=nz, tau=tau_of_viscosity(u * diameter / reynolds),
                    x_boundary=XBoundary.inflow_outflow,
                    y_low=wall(WallKind.slip), y_high=wall(WallKind.slip),
                    z_low=wall(WallKind.slip), z_high=wall(WallKind.slip), inlet_ux=u)
    centre = (upstream * diameter, 0.5 * (ny - 1) + 0.25, 0.5 * (nz - 1) + 0.25)
    return c, M.sphere_mask(nx, ny, nz, centre, 0.5 * diameter)


def cylinder_setup(nx, ny, diameter, cx, cy, u, reynolds):
    """Cylinder channel (lbm_test_support.h:146-167)."""
    c = Lbm2DConfig(nx=nx, ny=ny, tau=tau_of_viscosity(u * diameter / reynolds),
                    x_boundary=XBoundary.inflow_outflow, bottom=wall(WallKind.slip),
                    top=wall(WallKind.slip), inlet_ux=u)
    return c, M.circle_mask(nx, ny, cx, cy, 0.5 * diameter)


def copy_config(c):
    import copy
    return copy.deepcopy(c)


# D3Q19 tables (d3q19.h:15-36) for the test-side probes.
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def _stress(f):
    rho = float(np.sum(f))
    u = np.array([np.sum(CX * f), np.sum(CY * f), np.sum(CZ * f)]) / rho
    cu = CX * u[0] + CY * u[1] + CZ * u[2]
    feq = W19 * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * float(u @ u))
    neq = f - feq
    c = np.stack([CX, CY, CZ])
    return np.einsum("pi,si,i->ps", c, c, neq), rho


def closure_probe(initial, after, node, a, b, tau, constant, n=8):
    """Effective relaxation time of the first collision at `node` of a
    periodic n^3 box, and the Smagorinsky closure's prediction
    (lbm3d_test_support.h:171-239).  initial/after: (19, cells) arrays."""
    here = node[0] + n * (node[1] + n * node[2])
    before = np.empty(19)
    post = np.empty(19)
    for i in range(19):
        sx = (node[0] - CX[i]) % n
        sy = (node[1] - CY[i]) % n
        sz = (node[2] - CZ[i]) % n
        before[i] = initial[i, sx + n * (sy + n * sz)]
        post[i] = after[i, here]
    pi_before, rho = _stress(before)
    pi_after, _ = _stress(post)
    q2 = float(np.sum(pi_before * pi_before))
    measured = 1.0 / (1.0 - pi_after[a, b] / pi_before[a, b])
    predicted = 0.5 * (tau + math.sqrt(tau * tau + 18.0 * math.sqrt(2.0) * constant ** 2 * math.sqrt(q2) / rho))
    return measured, predicted
