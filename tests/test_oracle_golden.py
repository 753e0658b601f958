"""The C restatement of the oracle against the reference's own outputs.

tests/golden/reference_runs.npz holds what Orrery's CPU solvers (compiled from
the reference sources, tests/golden/make_golden.py) produce on small seeded
lattices covering every boundary option; the restatement must reproduce them
bit for bit.  Where oracle/_ref is built, the two are also compared directly.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "reference_runs.npz"))

import sys  # noqa: E402
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

CASES3D = {name: (steps, spec) for name, steps, spec in cases.lattice3d_cases()}
CASES2D = {name: (steps, spec) for name, steps, spec in cases.lattice2d_cases()}


@pytest.mark.parametrize("name", sorted(CASES3D))
def test_restated_d3q19_matches_reference_bitwise(name):
    steps, (cfg, mask, init, inlet) = CASES3D[name]
    o = O.Restated3D(cfg, mask.solid, mask.distance)
    if init is not None:
        o.initialize(*init)
    if inlet is not None:
        o.set_inlet_velocity(inlet)
    o.step(steps)
    assert np.array_equal(o.populations(), GOLDEN[f"{name}/populations"])
    rho, ux, uy, uz = o.macroscopic()
    for key, arr in (("rho", rho), ("ux", ux), ("uy", uy), ("uz", uz)):
        assert np.array_equal(arr, GOLDEN[f"{name}/{key}"]), key
    assert np.array_equal(o.force(), GOLDEN[f"{name}/force"])
    assert o.mass() == GOLDEN[f"{name}/mass"][0]
    cell, d, q = o.links()
    assert np.array_equal(cell, GOLDEN[f"{name}/link_cell"])
    assert np.array_equal(d, GOLDEN[f"{name}/link_dir"])
    assert np.array_equal(q, GOLDEN[f"{name}/link_q"])


@pytest.mark.parametrize("name", sorted(CASES2D))
def test_restated_d2q9_matches_reference_bitwise(name):
    steps, (cfg, mask, init) = CASES2D[name]
    o = O.Restated2D(cfg, mask.solid)
    if init is not None:
        o.initialize(*init)
    o.step(steps)
    assert np.array_equal(o.populations(), GOLDEN[f"{name}/populations"])
    rho, ux, uy = o.macroscopic()
    assert np.array_equal(rho, GOLDEN[f"{name}/rho"])
    assert np.array_equal(ux, GOLDEN[f"{name}/ux"])
    assert np.array_equal(o.force(), GOLDEN[f"{name}/force"])


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built here")
def test_restated_matches_built_reference_on_a_larger_lattice():
    """Direct comparison with the reference library where it is built."""
    from helpers import copy_config, sphere_channel
    from orrery_b200.lbm3d import Smagorinsky, SolidWall
    cfg, mask = sphere_channel(48, 24, 24, 8.0, 2.0, 0.05, 50.0)
    cfg = copy_config(cfg)
    cfg.smagorinsky = Smagorinsky(True, 0.12)
    cfg.solid_wall = SolidWall.interpolated
    a = O.Restated3D(cfg, mask.solid, mask.distance)
    b = O.Reference3D(cfg, mask.solid, mask.distance)
    a.step(40)
    b.step(40)
    assert np.array_equal(a.populations(), b.populations())
    assert np.array_equal(a.force(), b.force())
