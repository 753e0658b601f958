"""The reference's drag-table client on the CUDA solver, one point after
another and all points served together.

1. ``atmo::sample_cd_table`` (src/atmo/cd_sampling.cpp:98-120), compiled
   unmodified into the adapter harness, with the lattice Boltzmann solver
   forced and a factory of the reference's LbmAeroSolver3D on the CUDA
   solver: one adapter solve per Mach number (a 2 cm sphere, Re 40..100 over
   the table, the adapter's defaults: interpolated wall, sponge, gradual
   start, convective outlet), one after another.
2. The same points' lattice problems, as the adapter's setup builds them,
   submitted to one server at once (drag_table.serve_cd_table: fixed-length
   runs with the gradual start and the adapter's averaging window).

Bar: the served table's Cd at every Mach within 1e-4 relative of the
reference loop's (both run the binary32 CUDA step; the served run's inlet
ramp values are planned on the host by the adapter's own rule).
"""
import math

import pytest

from orrery_b200 import drag_table as D
from orrery_b200.lbm3d import Lbm3DConfig

pytestmark = pytest.mark.gpu

MACH = [0.02, 0.03, 0.04, 0.05]
TEMPERATURE = 288.15


def _oracle():
    from oracle import oracle as O
    if not O.adapter_available():
        pytest.skip("adapter harness not built (needs the reference tree at build time)")
    return O


def case(O):
    v, t = O.reference_mesh("sphere", 0.01, 32, 0.1)
    # speed of sound 340.3 m/s: 6.8 .. 17 m/s, Re = 1.2 U 0.02 / 4.08e-3 = 40 .. 100
    params = dict(length=0.02, area=0.25 * math.pi * 0.02 ** 2, density=1.2, viscosity=4.08e-3,
                  cells_per_length=10.0, lattice_velocity=0.05, upstream=2.0, downstream=4.0, width=4.0,
                  duration=5.0, average_window=2.0, steps_per_call=250)
    return v, t, params


def test_served_drag_table_matches_the_reference_loop():
    O = _oracle()
    v, t, p = case(O)
    ref = O.reference_cd_table(v, t, MACH, temperature=TEMPERATURE, storage=0, **p)
    assert [r["mach"] for r in ref] == MACH
    for r in ref:
        assert r["cd"] > 0 and r["table_cd"] == r["cd"]
    problems = []
    for m in MACH:
        q = O.reference_cd_point_problem(v, t, m, temperature=TEMPERATURE, **p)
        problems.append(D.LatticeProblem(
            mach=m, config=Lbm3DConfig.from_c(q["config"]), solid=q["solid"], distance=q["distance"],
            total_steps=int(q["total_steps"]), window_samples=int(q["window_samples"]),
            ramp_steps=q["ramp_steps"], area=q["area_lattice"], length=q["length_lattice"],
            sample_every=int(q["sample_every"])))
    served = D.serve_cd_table(problems, storage="f32")
    table = served["table"]
    stats = served["stats"]
    print(f"reference loop {ref[-1]['table_seconds']:.2f} s, served {stats['busy_seconds']:.2f} s busy, "
          f"{stats['mean_active']:.1f} solves resident on average, rounds of {served['chunk_steps']} steps")
    for r, (m, cd) in zip(ref, table.samples):
        print(f"Mach {m}: reference Cd {r['cd']!r}, served {cd!r}")
        assert abs(cd - r["cd"]) <= 1e-4 * abs(r["cd"]), (m, cd, r["cd"])
        assert table.cd(m) == cd
    assert stats["mean_active"] > 1.0   # the points ran together
    assert all(pt["steps"] == pr.total_steps for pt, pr in zip(served["points"], problems))
