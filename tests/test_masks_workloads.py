"""Mask builders against the reference's, seeded inputs and coefficients."""
import math
import os
import sys

import numpy as np

from orrery_b200 import masks as M
from orrery_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "golden", "reference_runs.npz"))


def test_sphere_masks_match_the_reference_bitwise():
    for name, (nx, ny, nz, centre, r) in cases.sphere_masks().items():
        m = M.sphere_mask(nx, ny, nz, centre, r)
        assert np.array_equal(m.solid, GOLDEN[f"mask/{name}/solid"])
        assert np.array_equal(m.distance, GOLDEN[f"mask/{name}/distance"])


def test_box_masks_match_the_reference_bitwise():
    for name, (nx, ny, nz, lo, hi) in cases.box_masks().items():
        m = M.box_mask(nx, ny, nz, lo, hi)
        assert np.array_equal(m.solid, GOLDEN[f"mask/{name}/solid"])
        assert np.array_equal(m.distance, GOLDEN[f"mask/{name}/distance"])


def test_circle_masks_match_the_reference_bitwise():
    for name, (nx, ny, cx, cy, r) in cases.circle_masks().items():
        assert np.array_equal(M.circle_mask(nx, ny, cx, cy, r).solid, GOLDEN[f"mask/{name}/solid"])


def test_noise_is_seeded_bounded_and_uncorrelated():
    a = W.uniform_noise(1, 100000, 0, 1e-3)
    b = W.uniform_noise(1, 100000, 0, 1e-3)
    c = W.uniform_noise(2, 100000, 0, 1e-3)
    d = W.uniform_noise(1, 100000, 1, 1e-3)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    assert np.max(np.abs(a)) <= 1e-3
    assert abs(np.mean(a)) < 1e-5
    assert abs(np.corrcoef(a, d)[0, 1]) < 0.02
    assert abs(np.std(a) - 1e-3 / math.sqrt(3)) < 1e-5


def test_sphere_workload_sizes():
    w = W.sphere3d(seed=1, nx=64, ny=32, nz=32, diameter=8.0)
    assert w.config.cells == 64 * 32 * 32
    assert abs(w.config.tau - (0.5 + 3 * 0.05 * 8 / 200)) < 1e-15
    fluid = w.mask.solid == 0
    assert np.all(w.ux[~fluid] == 0) and np.all(np.abs(w.ux[fluid] - 0.05) <= 1e-3)


def test_ellipsoid_and_capsule_masks_are_closed_bodies():
    e = M.ellipsoid_mask(96, 48, 48, (24.0, 24.0, 24.0), (12.0, 6.0, 6.0), math.radians(10))
    vol = np.count_nonzero(e.solid)
    assert abs(vol - 4 / 3 * math.pi * 12 * 6 * 6) / vol < 0.05
    c = M.sphere_cone_mask(96, 48, 48, (12.0, 24.0, 24.0), 10.0, math.radians(30), 3.0)
    assert np.count_nonzero(c.solid) > 0
    assert c.solid.reshape(48, 48, 96)[24, 24, 11] == 0 and c.solid.reshape(48, 48, 96)[24, 24, 14] == 1


def test_coefficients():
    q = 0.5 * 0.05 ** 2
    c = W.coefficients3d([q * 10.0, q * 2.0, 0.0], [0.0, 0.0, q * 10.0 * 4.0], 0.05, 10.0, 4.0)
    assert math.isclose(c["cd"], 1.0) and math.isclose(c["cl"], 0.2) and math.isclose(c["cm"], 1.0)
    c2 = W.coefficients2d(q * 32.0, -q * 3.2, 0.05, 32.0)
    assert math.isclose(c2["cd"], 1.0) and math.isclose(c2["cl"], -0.1)
