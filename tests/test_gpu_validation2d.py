"""Physical validation of the D2Q9 CUDA solver: the reference's cylinder case
(tests/aero_validation/lbm2d/test_cylinder.cpp:18-60 with cylinder_case.h):
Re 100, D 20 cells, inlet 8 D upstream, convective outlet 12 D downstream, a
20 D wide free-slip channel, a transverse bump behind the cylinder to start the
shedding, 26,000 steps with the force sampled every 10 and the last half
analysed.

Acceptance is the reference's literature bar: Strouhal number in [0.16, 0.20],
mean Cd in [1.2, 1.5] (over the analysed half and over the last period), lift
amplitude above 0.1, at least 5 cycles with periods within 5 percent, the
shedding analysed as the reference's dominant_oscillation does.
"""
import math

import numpy as np
import pytest

from orrery_b200 import masks as M
from orrery_b200 import solver as S
from orrery_b200.lbm3d import Lbm2DConfig, Outlet, WallKind, XBoundary, wall
from orrery_b200.workloads import coefficients2d, tau_of_viscosity

pytestmark = pytest.mark.gpu


def test_cylinder_sheds_at_the_literature_strouhal_number_and_drag():
    re, d, u = 100.0, 20.0, 0.05
    upstream, downstream, height, steps, every = 8.0, 12.0, 20.0, 26000, 10
    nx, ny = round((upstream + downstream) * d), round(height * d)
    # the reference's cylinder_setup leaves the outlet at Lbm2DConfig's
    # default, the convective outlet
    cfg = Lbm2DConfig(nx=nx, ny=ny, tau=tau_of_viscosity(u * d / re), x_boundary=XBoundary.inflow_outflow,
                      outlet=Outlet.convective, bottom=wall(WallKind.slip), top=wall(WallKind.slip),
                      inlet_ux=u)
    # the centre half a node off the channel axis (the discrete body is not
    # symmetric about it either)
    mask = M.circle_mask(nx, ny, upstream * d, 0.5 * (ny - 1) + 0.5, 0.5 * d)
    s = S.make_gpu_solver(cfg, mask)
    # free stream plus a transverse bump of 10 percent of U one diameter behind
    # the cylinder
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    bx, by = upstream * d + d, 0.5 * (ny - 1)
    rho = np.ones(nx * ny)
    ux = np.full(nx * ny, u)
    uy = (0.1 * u * np.exp(-((x - bx) ** 2 + (y - by) ** 2) / (d * d))).reshape(-1)
    s.initialize(rho, ux, uy)
    t, cd, cl = [], [], []
    for k in range(steps // every):
        s.step(every)
        f = s.force()
        c = coefficients2d(f.x, f.y, u, d)
        t.append((k + 1) * every)
        cd.append(c["cd"])
        cl.append(c["cl"])
    t, cd, cl = np.array(t, float), np.array(cd), np.array(cl)
    late = t >= 0.5 * steps
    tl, cdl, cll = t[late], cd[late], cl[late]
    # Shedding from the lift as the reference's dominant_oscillation defines it
    # (force_history.cpp:49-100): upward crossings of the mean, each counted
    # only after the signal was a quarter of its range below the mean; the
    # period from the first to the last crossing, the spread as (longest -
    # shortest) / period.
    mean = cll.mean()
    band = 0.25 * (cll.max() - cll.min())
    crossings, armed = [], False
    for k in range(1, len(tl)):
        a, b = cll[k - 1] - mean, cll[k] - mean
        if a < -band:
            armed = True
        if armed and a < 0.0 <= b:
            crossings.append(tl[k - 1] + a / (a - b) * (tl[k] - tl[k - 1]))
            armed = False
    periods = np.diff(crossings)
    period = (crossings[-1] - crossings[0]) / len(periods)
    strouhal = d / (u * period)
    spread = (periods.max() - periods.min()) / period
    mean_cd = cdl.mean()
    cd_last = cdl[tl >= tl[-1] - period].mean()
    amplitude = 0.5 * (cll.max() - cll.min())
    print(f"measured: cylinder Re {re:g} D {d:g} grid {nx}x{ny} steps {steps}: St {strouhal:.4f}, "
          f"mean Cd {mean_cd:.4f}, Cd over the last period {cd_last:.4f}, Cl amplitude {amplitude:.4f}, "
          f"cycles {len(periods)}, period spread {spread:.4f}")
    assert len(periods) >= 5
    assert spread < 0.05
    assert 0.16 <= strouhal <= 0.20
    assert 1.2 <= mean_cd <= 1.5
    assert 1.2 <= cd_last <= 1.5
    assert amplitude > 0.1
    assert math.isfinite(mean_cd)
