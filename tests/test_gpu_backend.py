"""The backend seam: the reference's own GPU driver, GpuLbm3D
(src/aero/lbm3d/lbm3d_gpu.cpp, its make_gpu_solver), compiled unmodified into
the harness library, runs its lbm_d3q19_step / _moments / _force dispatches
on the CUDA compute backend (orrery_b200/adapter/compute_backend_cuda.cpp,
the IComputeBackend of src/aero/compute/include/orrery/aero/compute/
compute_backend.h:94-129).

The cases and bars are the reference's GPU-vs-CPU comparisons
(tests/aero/lbm3d/test_lbm3d_gpu.cpp:196-275, its compare() at :56-75): the
same lattice on the reference's CPU solver and on the driver, velocity (and
where the reference checks them, populations and force x) within 1e-4
relative; and a uniform stream between co-moving walls stays uniform to 1e-4
at densities 0.7 and 2.
"""
import math

import numpy as np
import pytest

from helpers import (couette3d_config, duct_config, l2_relative, poiseuille3d_config,
                     sphere_channel, uniform_state_error, velocity_l2)
from orrery_b200 import masks as M
from orrery_b200.lbm3d import Outlet, Smagorinsky, SolidWall, WallKind, periodic_box, wall

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle as O
    if not (O.backend_available() and O.reference_available()):
        pytest.skip("backend harness not built (needs the reference tree at build time)")
    return O


def compare(O, config, mask, steps):
    """compare() of test_lbm3d_gpu.cpp:56-75 with the CUDA backend."""
    solid = mask.solid
    cpu = O.Reference3D(config, solid, mask.distance)
    cpu.initialize()
    cpu.step(steps)
    _, cux, cuy, cuz = cpu.macroscopic()
    fc = cpu.force()
    pc = cpu.populations()
    cpu.close()
    g = O.reference_gpu_driver_solve(config, solid, mask.distance, steps=steps)
    assert g["executes_kernels"] and g["steps"] == steps
    assert g["tables_built"] == 1          # one node-code buffer, tables kept over every dispatch
    assert g["dispatches"] >= steps + 1    # every step and the moments (and the force, with links) on the CUDA backend
    out = {
        "velocity": velocity_l2([g["ux"], g["uy"], g["uz"]], [cux, cuy, cuz], solid),
        "populations": l2_relative(g["populations"], pc),
        "force_x": abs(g["force"][0] - fc[0]) / abs(fc[0]) if fc[0] != 0 else abs(g["force"][0]),
    }
    print(f"measured: CUDA backend vs CPU after {steps} steps: {out}")
    return out


def test_analytic_flows():
    O = _oracle()
    cases = [(poiseuille3d_config(4, 32, 4, 0.8, 1e-6), (4, 32, 4)),
             (duct_config(4, 20, 20, 0.8, 1e-6), (4, 20, 20)),
             (couette3d_config(4, 4, 16, 0.8, 0.02), (4, 4, 16))]
    for cfg, dims in cases:
        mask = M.fluid_mask_3d(*dims)
        r = compare(O, cfg, mask, 4000)
        assert r["velocity"] < 1e-4, r


@pytest.mark.parametrize("variant", ["bgk", "les", "interpolated", "extrapolation_periodic_y"])
def test_laminar_sphere_channel(variant):
    O = _oracle()
    cfg, mask = sphere_channel(64, 32, 32, 8.0, 2.5, 0.05, 20.0)
    if variant == "les":
        cfg.smagorinsky = Smagorinsky(True, 0.1)
    elif variant == "interpolated":
        cfg.solid_wall = SolidWall.interpolated
    elif variant == "extrapolation_periodic_y":
        cfg.outlet = Outlet.extrapolation
        cfg.y_low = wall(WallKind.periodic)
        cfg.y_high = wall(WallKind.periodic)
    r = compare(O, cfg, mask, 800)
    assert r["velocity"] < 1e-4, r
    assert r["force_x"] < 1e-4, r
    if variant == "bgk":
        assert r["populations"] < 1e-4, r


def test_links_with_unusable_wall_distances():
    """Distances spoilt on the front half of the body (infinite on the fluid
    side) and on its rear half (positive inside): those links take the halfway
    wall (test_lbm3d_gpu.cpp:241-275)."""
    O = _oracle()
    cfg, mask = sphere_channel(48, 24, 24, 8.0, 2.0, 0.05, 20.0)
    cfg.solid_wall = SolidWall.interpolated
    centre = 2.0 * 8.0
    d = mask.distance.reshape(24, 24, 48).copy()
    s = mask.solid.reshape(24, 24, 48)
    front = (np.arange(48) < centre)[None, None, :]
    d[front & (s == 0)] = math.inf
    d[~front & (s != 0)] = 1.0
    mask.distance = d.reshape(-1)
    r = compare(O, cfg, mask, 400)
    assert r["velocity"] < 1e-4 and r["populations"] < 1e-4 and r["force_x"] < 1e-4, r


@pytest.mark.parametrize("rho", [0.7, 2.0])
def test_uniform_stream_between_co_moving_walls(rho):
    O = _oracle()
    cfg = periodic_box(4, 8, 8, 0.7)
    u = 0.03
    for name in ("y_low", "y_high", "z_low", "z_high"):
        setattr(cfg, name, wall(WallKind.no_slip, u))
    n = cfg.cells
    fields = (np.full(n, rho), np.full(n, u), np.zeros(n), np.zeros(n))
    g = O.reference_gpu_driver_solve(cfg, np.zeros(n, np.uint8), None, fields=fields, steps=300)
    worst = uniform_state_error(g["density"], g["ux"], g["uy"], g["uz"], rho, (u, 0.0, 0.0), u)
    print(f"measured: CUDA backend co-moving walls at density {rho}: {worst}")
    assert worst < 1e-4


def test_backend_refuses_bad_calls():
    O = _oracle()
    n, text = O.reference_backend_refusals()
    assert n == 5, text


def test_force_over_more_links_than_one_grid_dimension():
    """The driver's force dispatch for more links than 65535 groups of 64
    reach in one dimension (test_lbm3d_gpu_driver.cpp:93-156: a periodic
    128 x 128 x 66 box, fluid where x and y are even, 16 links per fluid
    node, 4,325,376 in all) tiles the links into rows; on the CUDA backend
    every link must be summed once.  Here the fluid moves (seeded velocities),
    so the force is not zero, and it must match the reference CPU solver's
    after one step."""
    O = _oracle()
    nx, ny, nz = 128, 128, 66
    cfg = periodic_box(nx, ny, nz, 0.6)
    mask = M.fluid_mask_3d(nx, ny, nz)
    x = np.arange(nx)[None, None, :]
    y = np.arange(ny)[None, :, None]
    solid = np.broadcast_to(~((x % 2 == 0) & (y % 2 == 0)), (nz, ny, nx)).astype(np.uint8).reshape(-1)
    mask.solid = solid
    rng = np.random.default_rng(17)
    n = cfg.cells
    fields = (1.0 + 1e-3 * rng.standard_normal(n), 0.02 * rng.standard_normal(n),
              0.02 * rng.standard_normal(n), 0.02 * rng.standard_normal(n))
    cpu = O.Reference3D(cfg, solid, None)
    links = len(cpu.links()[0])
    cpu.initialize(*fields)
    cpu.step(1)
    fc = np.asarray(cpu.force())
    cpu.close()
    assert links == nx * ny * nz // 4 * 16 and links > 65535 * 64
    g = O.reference_gpu_driver_solve(cfg, solid, None, fields=fields, steps=1)
    err = np.abs(np.asarray(g["force"]) - fc[:3]).max() / np.abs(fc[:3]).max()
    err_m = np.abs(np.asarray(g["moment"]) - fc[3:]).max() / np.abs(fc[3:]).max()
    print(f"measured: CUDA backend force over {links} links vs CPU: force {err:.2e}, moment {err_m:.2e} "
          f"of the largest component")
    assert err < 1e-4 and err_m < 1e-4
