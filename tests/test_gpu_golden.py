"""The CUDA path against the reference's own outputs (tests/golden).

For every golden lattice the binary64 device form must reproduce Orrery's CPU
solver bit for bit (populations and moments; force and moment to the rounding
of a reordered sum), and the binary32 form must stay within the relative-L2
tolerance of the plain path (1e-5 on populations, 1e-4 on force).
"""
import os
import sys

import numpy as np
import pytest

from helpers import l2_relative
from orrery_b200 import solver as S

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "golden", "reference_runs.npz"))
C3 = {n: (s, spec) for n, s, spec in cases.lattice3d_cases()}
C2 = {n: (s, spec) for n, s, spec in cases.lattice2d_cases()}


def run3(name, storage):
    steps, (cfg, mask, init, inlet) = C3[name]
    g = S.make_gpu_solver(cfg, mask, storage=storage)
    if init is not None:
        g.initialize(*init)
    if inlet is not None:
        g.set_inlet_velocity(inlet)
    g.step(steps)
    return g


@pytest.mark.parametrize("name", sorted(C3))
def test_d3q19_binary64_equals_reference(name):
    g = run3(name, "f64")
    assert np.array_equal(g.populations(), GOLDEN[f"{name}/populations"])
    m = g.macroscopic()
    assert np.array_equal(m.density, GOLDEN[f"{name}/rho"])
    assert np.array_equal(m.velocity_x, GOLDEN[f"{name}/ux"])
    assert np.array_equal(m.velocity_y, GOLDEN[f"{name}/uy"])
    assert np.array_equal(m.velocity_z, GOLDEN[f"{name}/uz"])
    f = g.force()
    ref = GOLDEN[f"{name}/force"]
    assert np.allclose(f.force, ref[:3], rtol=0, atol=1e-12)
    assert np.allclose(f.moment, ref[3:], rtol=0, atol=1e-10)
    assert g.mass() == pytest.approx(GOLDEN[f"{name}/mass"][0], rel=1e-13)


@pytest.mark.parametrize("name", sorted(C3))
def test_d3q19_binary32_within_tolerance(name):
    g = run3(name, "f32")
    assert l2_relative(g.populations(), GOLDEN[f"{name}/populations"]) < 1e-5
    fx = g.force().force[0]
    ref = GOLDEN[f"{name}/force"][0]
    assert abs(fx - ref) <= 1e-4 * max(abs(ref), 1e-3)


@pytest.mark.parametrize("name", sorted(C2))
def test_d2q9_binary64_equals_reference(name):
    steps, (cfg, mask, init) = C2[name]
    g = S.make_gpu_solver(cfg, mask, storage="f64")
    g.initialize(*init)
    g.step(steps)
    assert np.array_equal(g.populations(), GOLDEN[f"{name}/populations"])
    f = g.force()
    ref = GOLDEN[f"{name}/force"]
    assert abs(f.x - ref[0]) < 1e-12 and abs(f.y - ref[1]) < 1e-12 and abs(f.moment - ref[2]) < 1e-10
