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


# ---- D2Q9: the reference's GpuLbm2D on the CUDA backend -------------------
# Cases and bars of the reference's 2D GPU-vs-CPU comparisons
# (tests/aero/lbm/test_lbm_gpu.cpp:83-120 compare(), 204-276), with the CUDA
# backend in place of the GL one.

def _fluid2(nx, ny):
    return np.zeros(nx * ny, np.uint8)


def _density_deviation_error(a, b, solid):
    """density_deviation_error of lbm_test_support.h:60-78."""
    keep = np.asarray(solid) == 0
    a, b = np.asarray(a)[keep], np.asarray(b)[keep]
    peak = float(np.max(np.abs(b - 1.0))) if b.size else 0.0
    diff = float(np.sum((a - b) ** 2))
    if b.size == 0 or peak == 0.0:
        return math.sqrt(diff)
    return math.sqrt(diff / b.size) / peak


def compare2(O, config, solid, steps, fields=None, via="backend"):
    """compare() of test_lbm_gpu.cpp:83-120 with the CUDA backend under the
    reference's GpuLbm2D (via "backend"), or with the C++ Lbm2DSolver adapter
    of orrery_b200/adapter/lbm2d_cuda.cpp (via "solver")."""
    cpu = O.Reference2D(config, solid)
    if fields is not None:
        cpu.initialize(*fields)
    cpu.step(steps)
    crho, cux, cuy = cpu.macroscopic()
    fc = cpu.force()
    pc = cpu.populations()
    cpu.close()
    if via == "backend":
        g = O.reference_gpu_driver_solve2d(config, solid, fields=fields, steps=steps)
        assert g["executes_kernels"] and g["steps"] == steps
        assert g["tables_built"] == 1      # one solid-flag buffer, tables kept over every dispatch
    else:
        g = O.reference_cuda2d_solve(config, solid, fields=fields, steps=steps)
        assert g["steps"] == steps
    out = {
        "velocity": velocity_l2([g["ux"], g["uy"]], [cux, cuy], solid),
        "density": _density_deviation_error(g["density"], crho, solid),
        "populations": l2_relative(g["populations"], pc),
        "force_x": abs(g["force"][0] - fc[0]) / abs(fc[0]) if fc[0] != 0 else abs(g["force"][0]),
    }
    print(f"measured: CUDA D2Q9 ({via}) vs CPU after {steps} steps: {out}")
    return out


@pytest.mark.parametrize("via", ["backend", "solver"])
def test_d2q9_analytic_flows(via):
    O = _oracle()
    from orrery_b200.lbm3d import Lbm2DConfig, XBoundary
    pois = Lbm2DConfig(nx=8, ny=64, tau=0.8, x_boundary=XBoundary.periodic, bottom=wall(WallKind.no_slip),
                       top=wall(WallKind.no_slip), body_force_x=1e-6)
    assert compare2(O, pois, _fluid2(8, 64), 4000, via=via)["velocity"] < 1e-4
    cou = Lbm2DConfig(nx=8, ny=32, tau=0.9, x_boundary=XBoundary.periodic, bottom=wall(WallKind.no_slip),
                      top=wall(WallKind.no_slip, 0.03))
    assert compare2(O, cou, _fluid2(8, 32), 4000, via=via)["velocity"] < 1e-4
    # Taylor-Green vortex on a periodic 64 x 64 box (taylor_green, :106-116)
    n, u0 = 64, 0.03
    box = Lbm2DConfig(nx=n, ny=n, tau=0.6, x_boundary=XBoundary.periodic, bottom=wall(WallKind.periodic),
                      top=wall(WallKind.periodic))
    k = 2.0 * math.pi / n
    y, x = np.meshgrid(np.arange(n, dtype=np.float64), np.arange(n, dtype=np.float64), indexing="ij")
    rho = 1.0 - 0.75 * u0 * u0 * (np.cos(2.0 * k * x) + np.cos(2.0 * k * y))
    ux = -u0 * np.cos(k * x) * np.sin(k * y)
    uy = u0 * np.sin(k * x) * np.cos(k * y)
    r = compare2(O, box, _fluid2(n, n), 2000, fields=(rho.reshape(-1), ux.reshape(-1), uy.reshape(-1)), via=via)
    assert r["velocity"] < 1e-4 and r["density"] < 1e-3, r


@pytest.mark.parametrize("rho", [1.0, 2.0, 0.7])
def test_d2q9_uniform_stream_between_co_moving_walls(rho):
    O = _oracle()
    from orrery_b200.lbm3d import Lbm2DConfig, XBoundary
    u = 0.02
    cfg = Lbm2DConfig(nx=4, ny=12, tau=0.8, x_boundary=XBoundary.periodic, bottom=wall(WallKind.no_slip, u),
                      top=wall(WallKind.no_slip, u))
    n = 4 * 12
    g = O.reference_gpu_driver_solve2d(cfg, _fluid2(4, 12), fields=(np.full(n, rho), np.full(n, u), np.zeros(n)),
                                       steps=200)
    worst = max(float(np.max(np.abs(g["density"] - rho) / rho)), float(np.max(np.abs(g["ux"] - u) / u)),
                float(np.max(np.abs(g["uy"]) / u)))
    print(f"measured: CUDA backend D2Q9 co-moving walls at density {rho}: {worst}")
    assert worst < 1e-4


@pytest.mark.parametrize("via", ["backend", "solver"])
@pytest.mark.parametrize("les", [False, True])
def test_d2q9_cylinder_channel(les, via):
    """Re 100, D 10 at (50, 50.5) of 200 x 100: Zou-He inlet, extrapolation
    outlet, slip sides, bounce-back and momentum exchange, with and without
    the LES closure (C 0.17), 4000 steps (test_lbm_gpu.cpp:259-276)."""
    O = _oracle()
    from helpers import cylinder_setup
    from orrery_b200.lbm3d import Smagorinsky
    cfg, mask = cylinder_setup(200, 100, 10.0, 50.0, 50.5, 0.05, 100.0)
    if les:
        cfg.smagorinsky = Smagorinsky(True, 0.17)
    r = compare2(O, cfg, mask.solid, 4000, via=via)
    assert r["velocity"] < 1e-4 and r["force_x"] < 1e-4, r


def test_d2q9_adapter_on_the_cuda_backend():
    """The reference's 2D adapter with its backend option set to the CUDA
    backend (test_lbm_gpu.cpp:278-311): Cd within 1e-4 of the CPU solver's,
    the same iterations and surface samples."""
    O = _oracle()
    r = O.reference_adapter2d_on_backend()
    print(f"measured: 2D adapter Cd CPU {r['cd_cpu']!r}, CUDA backend {r['cd_gpu']!r}")
    assert r["cd_gpu"] == pytest.approx(r["cd_cpu"], rel=1e-4)
    assert r["iterations_gpu"] == r["iterations_cpu"]
    assert r["cp_gpu"] == r["cp_cpu"] > 0


def test_d3q19_adapter_on_the_cuda_backend():
    """The reference's 3D adapter, unmodified, with its backend option set to
    the CUDA backend, so its own GPU driver runs the lattice
    (test_lbm3d_gpu.cpp:291-324): Cd within 1e-4 of the CPU solver's and the
    same iterations."""
    O = _oracle()
    r = O.reference_adapter3d_on_backend()
    print(f"measured: 3D adapter Cd CPU {r['cd_cpu']!r}, GPU driver on the CUDA backend {r['cd_gpu']!r}")
    assert abs(r["cd_gpu"] - r["cd_cpu"]) / r["cd_cpu"] < 1e-4
    assert r["iterations_gpu"] == r["iterations_cpu"]


def test_smagorinsky_closure_through_the_driver():
    """The closure relaxes a manufactured shear at the predicted rate on the
    driver's binary32 populations (test_lbm3d_gpu.cpp:168-195: tau 0.52,
    C 0.4, shear 0.01 along every pair of axes): the effective relaxation
    time of one collision within 2% of tau_eff - tau."""
    O = _oracle()
    from helpers import closure_probe
    tau, gamma, cconst = 0.52, 0.01, 0.4
    n = 8
    coords = [np.tile(np.arange(n), n * n), np.tile(np.repeat(np.arange(n), n), n), np.repeat(np.arange(n), n * n)]
    worst = 0.0
    for a in range(3):
        for b in range(3):
            if a == b:
                continue
            cfg = periodic_box(n, n, n, tau)
            cfg.smagorinsky = Smagorinsky(True, cconst)
            cells = cfg.cells
            u = [np.zeros(cells), np.zeros(cells), np.zeros(cells)]
            u[a] = gamma * (coords[b] - 3.5)
            fields = (np.ones(cells), *u)
            solid = np.zeros(cells, np.uint8)
            before = O.reference_gpu_driver_solve(cfg, solid, fields=fields, steps=0)["populations"]
            after = O.reference_gpu_driver_solve(cfg, solid, fields=fields, steps=1)["populations"]
            for k in (1, 3, 6):
                node = [2, 5, 4]
                node[b] = k
                measured, predicted = closure_probe(before.reshape(19, cells), after.reshape(19, cells), node,
                                                    a, b, tau, cconst)
                rel = abs(measured - predicted) / (predicted - tau)
                worst = max(worst, rel)
                assert rel < 0.02, (a, b, k, measured, predicted)
    print(f"measured: closure through the driver on the CUDA backend, worst |tau_eff - closure| / "
          f"(closure - tau) {worst:.2e}")


def test_reference_benchmark_goals_through_the_driver():
    """The reference's own GPU benchmark (tests/bench/aero/bench_lbm_gpu.cpp:
    D3Q19 128^3 sphere channel, D2Q9 2048 x 1024 cylinder, BGK and
    Smagorinsky; 50 warm-up steps, 1000 timed) with its own GPU driver on the
    CUDA backend meets the goals the benchmark sets (at least 60 and 200
    steps/s).  The rates include the driver's host loop (one dispatch per
    step)."""
    O = _oracle()
    from orrery_b200 import workloads as W
    goals = {3: 60.0, 2: 200.0}
    for case in W.reference_benchmarks():
        rate = O.reference_driver_rate(case.config, case.mask.solid)
        dim = 3 if case.name.startswith("sphere3d") else 2
        print(f"measured: reference benchmark {case.name} through its GPU driver on the CUDA backend: "
              f"{rate:.0f} steps/s ({rate * case.cells / 1e6:.0f} MLUPS; published on its GL backend "
              f"{case.published_steps_per_s} steps/s)")
        assert rate >= goals[dim]
