"""The reference's own 3D adapter, LbmAeroSolver3D, end to end on the CUDA
solver (oracle/_ref/libref_adapter.so: the adapter compiled unmodified, its
GPU branch routed through the Lbm3DSolver seam to make_cuda_solver of
orrery_b200/adapter/lbm3d_cuda.cpp).

The bar is the reference's own (tests/aero/lbm3d/test_lbm3d_gpu.cpp:291-324,
"The 3D IAeroSolver adapter runs on the GPU backend"): the same adapter solve
on the CPU solver and on the GPU solver gives Cd within 1e-4 relative and the
same number of iterations.  The binary64 device form gives the CPU solver's
force to the rounding of its summation order.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle as O
    if not O.adapter_available():
        pytest.skip("adapter harness not built (needs the reference tree at build time)")
    return O


def sphere_case(O):
    """The reference test's case: a 2 cm sphere at Re 50, 10 cells per
    diameter, 2 / 4 / 4 diameters upstream / downstream / wide, 5 convective
    times with a 2-time average, interpolated wall, sponge and gradual start
    (the adapter's defaults)."""
    v, t = O.reference_mesh("sphere", 0.01, 32, 0.1)
    params = dict(length=0.02, area=0.25 * math.pi * 0.02 ** 2, speed=0.1, density=1000.0,
                  viscosity=1000.0 * 0.1 * 0.02 / 50.0, cells_per_length=10.0, lattice_velocity=0.05,
                  upstream=2.0, downstream=4.0, width=4.0, duration=5.0, average_window=2.0, steps_per_call=1000)
    return v, t, params


def test_adapter_runs_on_the_cuda_solver():
    O = _oracle()
    v, t, p = sphere_case(O)
    cpu = O.reference_adapter_run(v, t, "cpu", fields=True, **p)
    gpu = O.reference_adapter_run(v, t, "cuda", 0, fields=True, **p)
    print(f"measured: 3D adapter Cd CPU {cpu['cd']!r}, CUDA {gpu['cd']!r}; lattice "
          f"{int(cpu['nx'])}x{int(cpu['ny'])}x{int(cpu['nz'])}, {int(cpu['lattice_steps'])} steps; "
          f"{cpu['seconds']:.2f} s CPU, {gpu['seconds']:.2f} s CUDA")
    assert (gpu["nx"], gpu["ny"], gpu["nz"]) == (cpu["nx"], cpu["ny"], cpu["nz"])
    assert gpu["iterations"] == cpu["iterations"]
    # the result's wall pressure and velocity field (update_result), read back
    # through the solver's macroscopic(): the same samples, binary32 close
    assert len(gpu["cp"]) == len(cpu["cp"]) > 0
    assert np.max(np.abs(gpu["cp"] - cpu["cp"])) < 1e-3 * np.max(np.abs(cpu["cp"]))
    assert gpu["velocity"].shape == cpu["velocity"].shape
    assert np.max(np.abs(gpu["velocity"] - cpu["velocity"])) < 1e-4 * p["speed"]
    assert gpu["lattice_steps"] == cpu["lattice_steps"]
    assert abs(gpu["cd"] - cpu["cd"]) / abs(cpu["cd"]) < 1e-4, (gpu["cd"], cpu["cd"])


def test_adapter_binary64_form_matches_cpu_solver():
    O = _oracle()
    v, t, p = sphere_case(O)
    cpu = O.reference_adapter_run(v, t, "cpu", **p)
    f64 = O.reference_adapter_run(v, t, "cuda", 3, **p)   # ORR_STORAGE_F64
    print(f"measured: 3D adapter Cd CPU {cpu['cd']!r}, CUDA binary64 {f64['cd']!r}")
    for k in ("cd", "cl", "cy", "cm"):
        assert abs(f64[k] - cpu[k]) <= 1e-10 * max(abs(cpu["cd"]), 1e-30), (k, f64[k], cpu[k])


def test_adapter_halfway_les_and_incidence():
    """Halfway wall, the LES closure, angle of attack and sideslip (the wind
    frame rotates the body), a NACA 2412 wing."""
    O = _oracle()
    v, t = O.reference_mesh("naca_wing", "2412", 0.02, 0.04, 24, 8)
    p = dict(length=0.02, area=0.02 * 0.04, speed=0.1, density=1000.0, viscosity=1000.0 * 0.1 * 0.02 / 400.0,
             angle_of_attack=math.radians(6.0), sideslip=math.radians(3.0), cells_per_length=12.0,
             lattice_velocity=0.05, upstream=1.5, downstream=3.0, width=3.0, duration=4.0, average_window=1.5,
             steps_per_call=500, wall=0, les=1)
    cpu = O.reference_adapter_run(v, t, "cpu", **p)
    gpu = O.reference_adapter_run(v, t, "cuda", 0, **p)
    print(f"measured: wing Cd CPU {cpu['cd']!r}, CUDA {gpu['cd']!r}; Cl CPU {cpu['cl']!r}, CUDA {gpu['cl']!r}")
    assert gpu["iterations"] == cpu["iterations"]
    assert abs(gpu["cd"] - cpu["cd"]) / abs(cpu["cd"]) < 1e-4, (gpu["cd"], cpu["cd"])
    assert abs(gpu["cl"] - cpu["cl"]) < 1e-4 * abs(cpu["cd"]), (gpu["cl"], cpu["cl"])


def test_adapter_with_the_device_voxelizer():
    """The adapter with the reference's voxel_grid.cpp replaced by the device
    voxelizer (orrery_b200/adapter/voxel_grid_cuda.cpp): the same mask and
    wall distances, so the CPU solver's solve is the same bit for bit, and
    the whole pipeline on the device meets the reference test's bar."""
    O = _oracle()
    v, t, p = sphere_case(O)
    ref = O.reference_adapter_run(v, t, "cpu", voxelizer="cpu", **p)
    dev = O.reference_adapter_run(v, t, "cpu", voxelizer="device", **p)
    assert dev == {**ref, "seconds": dev["seconds"]}
    gpu = O.reference_adapter_run(v, t, "cuda", 0, voxelizer="device", **p)
    print(f"measured: adapter on the device end to end, Cd {gpu['cd']!r} (CPU {ref['cd']!r})")
    assert gpu["iterations"] == ref["iterations"]
    assert abs(gpu["cd"] - ref["cd"]) / abs(ref["cd"]) < 1e-4
