"""The C ABI library on the host: it loads without a GPU, exports every entry
point include/orrery_lbm.h declares, refuses configurations with the
reference's messages, and plans links like the reference.  No compute call
runs here."""
import ctypes
import os
import re
import sys

import numpy as np
import pytest

from orrery_b200 import _native, abi
from orrery_b200 import masks as M
from orrery_b200 import solver as S
from orrery_b200.lbm3d import Lbm3DConfig, periodic_box

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "golden", "reference_runs.npz"))


def declared_entry_points():
    with open(os.path.join(ROOT, "include", "orrery_lbm.h")) as fh:
        text = fh.read()
    return sorted(set(re.findall(r"ORR_API\s+[\w\s\*]*?\b(orr_\w+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    names = declared_entry_points()
    assert len(names) >= 30
    lib = _native.lib()
    for name in names:
        assert hasattr(lib, name), name
    # and the binding declares them all
    assert set(names) == set(_native.SIGNATURES)


def test_exports_only_the_abi():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", _native.library_path()], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("nm not available")
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.split()[-1].startswith("orr_")}
    assert exported == set(declared_entry_points())


def test_version_and_device_count_without_a_gpu():
    lib = _native.lib()
    assert b"sm_100a" in lib.orr_version()
    n = ctypes.c_int32(-1)
    assert lib.orr_device_count(ctypes.byref(n)) == abi.ORR_OK
    assert n.value >= 0


@pytest.mark.parametrize("dims", [3, 2])
def test_validation_messages_match_the_reference(dims):
    import json
    with open(os.path.join(HERE, "golden", "validation_messages.json")) as fh:
        expected = {(m["dims"], m["label"]): m["message"] for m in json.load(fh)}
    for label, cfg, mask in (cases.validation_cases3d() if dims == 3 else cases.validation_cases2d()):
        got = S.validate(cfg, mask) or ""
        assert got == expected[(dims, label)], label


def test_mach_guard_opt_in():
    cfg = periodic_box(8, 8, 8, 0.6)
    cfg.x_boundary = 1
    cfg.inlet_ux = 0.08
    mask = M.fluid_mask_3d(8, 8, 8)
    assert "lattice Mach number 0.138564" in S.validate(cfg, mask)
    assert S.validate(cfg, mask, allow_high_mach=True) is None


def test_binary32_refusals():
    mask = M.fluid_mask_3d(8, 8, 8)
    cfg = periodic_box(8, 8, 8, 0.50000001)
    assert "rounds to 1/2 in binary32" in S.validate(cfg, mask)
    assert S.validate(cfg, mask, storage="f64") is None  # binary64 kernels keep the viscosity
    cfg = periodic_box(8, 8, 8, 0.6)
    cfg.body_force_x = 1e39
    assert "outside the binary32 range" in S.validate(cfg, mask)


@pytest.mark.parametrize("name", [n for n, _, _ in cases.lattice3d_cases()])
def test_planned_links_match_the_reference(name):
    spec = {n: s for n, _, s in cases.lattice3d_cases()}[name]
    cfg, mask = spec[0], spec[1]
    cell, d, q, fluid, _ = S.plan3d(cfg, mask)
    assert np.array_equal(cell, GOLDEN[f"{name}/link_cell"])
    assert np.array_equal(d, GOLDEN[f"{name}/link_dir"])
    assert np.array_equal(q, GOLDEN[f"{name}/link_q"])
    assert fluid == int(np.count_nonzero(mask.solid == 0))


def test_create_refuses_before_allocating_without_a_device():
    cfg = periodic_box(8, 8, 8, 0.6)
    mask = M.fluid_mask_3d(8, 8, 8)
    if _device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(_native.LbmError) as e:
        S.make_gpu_solver(cfg, mask)
    assert e.value.status in (abi.ORR_ERR_NO_DEVICE, abi.ORR_ERR_CUDA)
    # an invalid configuration is refused with its reason first
    bad = periodic_box(8, 8, 8, 0.5)
    with pytest.raises(_native.LbmError) as e:
        S.make_gpu_solver(bad, mask)
    assert e.value.status == abi.ORR_ERR_INVALID
    assert "tau must be finite" in str(e.value)


def _device_count():
    n = ctypes.c_int32(0)
    _native.lib().orr_device_count(ctypes.byref(n))
    return n.value


def test_memory_estimate_counts_every_table():
    cfg = Lbm3DConfig(nx=128, ny=128, nz=128)
    cells = 128 ** 3
    f32 = S.memory_bytes(cfg, 0, 0, "f32")
    f16 = S.memory_bytes(cfg, 0, 0, "f16")
    f64 = S.memory_bytes(cfg, 0, 0, "f64")
    assert f32 >= cells * (2 * 19 * 4 + 1 + 4 + 16)
    # The two population buffers, plus their slack of 2 x 1024 values each.
    assert f32 - f16 == cells * 2 * 19 * 2 + 4 * 1024 * 2
    assert f64 > f32
    with pytest.raises(_native.LbmError):
        S.memory_bytes(Lbm3DConfig(nx=4, ny=4, nz=(1 << 60) + 1), 0, 0)


def test_server_refuses_bfloat16_before_touching_a_device():
    """Served solves promise Cd within 0.5% of binary64, which bfloat16
    storage misses; the refusal comes before any device call, so it holds
    without a GPU."""
    from orrery_b200.serve import Server
    with pytest.raises(_native.LbmError) as e:
        Server(storage="bf16")
    assert e.value.status == abi.ORR_ERR_INVALID
    assert "bfloat16" in str(e.value) and "0.5%" in str(e.value)


@pytest.mark.skipif(__import__("shutil").which("gcc") is None, reason="needs gcc")
def test_ctypes_records_match_the_header(tmp_path):
    """Every ctypes record of the Python binding has the size and field
    offsets of its C struct in include/orrery_lbm.h (a smaller record would
    let the library write past a Python buffer)."""
    import os
    import subprocess
    pairs = {"orr_wall": abi.CWall, "orr_lbm3d_config": abi.CLbm3DConfig, "orr_lbm2d_config": abi.CLbm2DConfig,
             "orr_force_links": abi.CForceLinks, "orr_kernel_info": abi.CKernelInfo,
             "orr_solver_options": abi.CSolverOptions, "orr_batch_schedule": abi.CBatchSchedule,
             "orr_serve_options": abi.CServeOptions, "orr_solve_request": abi.CSolveRequest,
             "orr_solve_result": abi.CSolveResult, "orr_serve_statistics": abi.CServeStatistics,
             "orr_grid_spec": abi.CGridSpec, "orr_mesh": abi.CMesh}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "orrery_lbm.h"', "int main(void) {"]
    for name, rec in pairs.items():
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in rec._fields_:
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "records.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "records"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    seen = {}
    for line in out:
        if line:
            name, field, value = line.split()
            seen[(name, field)] = int(value)
    for name, rec in pairs.items():
        assert seen[(name, "size")] == ctypes.sizeof(rec), name
        for field, _ in rec._fields_:
            assert seen[(name, field)] == getattr(rec, field).offset, (name, field)
