"""The host planner (orrery_b200/csrc/plan.cpp) under ThreadSanitizer and under
AddressSanitizer + UndefinedBehaviorSanitizer, on the CPU.

Validation (the NaN scan of the wall distances) and planning run on several
host threads for lattices of 2^20 cells or more; the planner splits the
lattice into z-slabs whose threads each fill their own rows of the per-cell
tables and keep their links in scan order.  The unit is compiled with g++
together with a small driver (tests/native/plan_sanitize_test.cpp) and run on
lattices above that size: halfway and interpolated walls, slip, periodic and
no-slip sides, one refused configuration.  Both instrumented builds must run
clean and print the same node counts and table digests, and their boundary
links must equal those of the library's own planner (orr_lbm3d_plan)."""
import ctypes
import os
import re
import shutil
import struct
import subprocess

import numpy as np
import pytest

from orrery_b200 import lbm3d as L3
from orrery_b200 import masks as M
from orrery_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def _cases():
    """(config, mask) pairs of at least 2^20 cells."""
    out = []
    w = W.sphere3d(seed=3, nx=128, ny=96, nz=96, diameter=24.0)
    out.append((w.config, w.mask))                                   # slip sides, halfway wall
    cfg = L3.Lbm3DConfig(**{**w.config.__dict__, "solid_wall": L3.SolidWall.interpolated})
    out.append((cfg, w.mask))                                        # interpolated wall (slots, fractions)
    cfg = L3.Lbm3DConfig(**{**w.config.__dict__,
                            "y_low": L3.Wall(L3.WallKind.periodic), "y_high": L3.Wall(L3.WallKind.periodic),
                            "z_low": L3.Wall(L3.WallKind.no_slip), "z_high": L3.Wall(L3.WallKind.no_slip, 0.01)})
    mask = M.sphere_mask(128, 96, 96, (40.0, 48.0, 20.0), 14.0)      # a body touching the face rows' sources
    out.append((cfg, mask))
    bad = M.SolidMask3D(128, 96, 96, w.mask.solid, w.mask.distance.copy())
    bad.distance[12345] = np.nan                                     # refused: NaN wall distance
    out.append((L3.Lbm3DConfig(**{**w.config.__dict__, "solid_wall": L3.SolidWall.interpolated}), bad))
    return out


def _write(path, cases):
    with open(path, "wb") as fh:
        for cfg, mask in cases:
            c = bytes(cfg.to_c())
            fh.write(struct.pack("<I", len(c)))
            fh.write(c)
            solid = np.ascontiguousarray(mask.solid, dtype=np.uint8).reshape(-1)
            fh.write(struct.pack("<Q", solid.size))
            fh.write(solid.tobytes())
            if mask.distance is None:
                fh.write(b"\x00")
            else:
                fh.write(b"\x01")
                fh.write(np.ascontiguousarray(mask.distance, np.float64).reshape(-1).tobytes())


def _build(tmp_path, name, flags):
    exe = str(tmp_path / name)
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-pthread", *flags,
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "orrery_b200", "csrc"),
           os.path.join(ROOT, "tests", "native", "plan_sanitize_test.cpp"),
           os.path.join(ROOT, "orrery_b200", "csrc", "plan.cpp"), "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def _run(exe, case_file, env):
    res = subprocess.run([exe, case_file], capture_output=True, text=True, timeout=900,
                         env=dict(os.environ, **env))
    assert res.returncode == 0, res.stdout + res.stderr
    assert "WARNING: ThreadSanitizer" not in res.stderr, res.stderr
    assert "ERROR: AddressSanitizer" not in res.stderr, res.stderr
    assert "runtime error" not in res.stderr, res.stderr
    lines = res.stdout.strip().splitlines()
    assert lines[-1] == "ok"
    return lines[:-1]


def _fnv1a(data: bytes, h: int = 1469598103934665603) -> int:
    for b in data:
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_planner_is_clean_under_thread_and_address_sanitizers(tmp_path):
    cases = _cases()
    case_file = str(tmp_path / "cases.bin")
    _write(case_file, cases)
    tsan = _run(_build(tmp_path, "plan_tsan", ["-fsanitize=thread"]), case_file,
                {"TSAN_OPTIONS": "halt_on_error=1"})
    asan = _run(_build(tmp_path, "plan_asan", ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined"]),
                case_file, {"ASAN_OPTIONS": "detect_leaks=1"})
    assert tsan == asan
    assert len(tsan) == len(cases)
    assert "refused" in tsan[-1] and "refused" not in " ".join(tsan[:-1])

    # The boundary links and node counts of the instrumented builds equal the
    # library's planner on the same inputs.
    try:
        from orrery_b200 import solver as S
        S.lib()
    except Exception as exc:          # library not built in this checkout
        pytest.skip(f"native library unavailable: {exc}")
    for k, (cfg, mask) in enumerate(cases[:-1]):
        cell, d, q, fluid, boundary = S.plan3d(cfg, mask)
        m = re.match(r"case (\d+) fluid (\d+) general (\d+) links (\d+) links_digest ([0-9a-f]+) ", tsan[k])
        assert m is not None, tsan[k]
        assert int(m.group(2)) == fluid
        assert int(m.group(3)) == boundary
        assert int(m.group(4)) == cell.size
        h = _fnv1a(np.ascontiguousarray(cell, np.uint32).tobytes())
        h = _fnv1a(np.ascontiguousarray(d, np.uint32).tobytes(), h)
        h = _fnv1a(np.ascontiguousarray(q, np.float64).tobytes(), h)
        assert int(m.group(5), 16) == h
