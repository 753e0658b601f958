"""Generates the golden fixtures of tests/golden from the reference itself.

Runs Orrery's own CPU solvers, compiled from the reference sources into
oracle/_ref by oracle/Makefile, on small seeded lattices and stores what they
produce: populations, moments, force and moment, mass and boundary links after
a number of steps; the refusal messages of validate(); and the reference's mask
builders.  The tests check the C restatement (oracle/lbm_oracle.c), the
package's mask builders and validation, and the CUDA path against these files.

    python tests/golden/make_golden.py      (needs oracle/_ref; writes tests/golden/*)
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402
from orrery_b200 import masks as M  # noqa: E402
from orrery_b200 import workloads as W  # noqa: E402
from orrery_b200.lbm3d import (Lbm2DConfig, Lbm3DConfig, Outlet, Smagorinsky, SolidWall, Sponge,  # noqa: E402
                               WallKind, XBoundary, periodic_box, tau_of_viscosity, wall)

import cases  # noqa: E402  (tests/golden/cases.py)


def config_to_dict(c) -> dict:
    out = {}
    for k, v in c.__dict__.items():
        if hasattr(v, "__dict__"):
            out[k] = {kk: (int(vv) if hasattr(vv, "value") else vv) for kk, vv in v.__dict__.items()}
        else:
            out[k] = int(v) if hasattr(v, "value") else v
    return out


def run3d(name: str, steps: int, cfg, mask, init=None, inlet=None) -> dict:
    ref = O.Reference3D(cfg, mask.solid, mask.distance)
    if init is not None:
        ref.initialize(*init)
    if inlet is not None:
        ref.set_inlet_velocity(inlet)
    ref.step(steps)
    rho, ux, uy, uz = ref.macroscopic()
    cell, d, q = ref.links()
    out = {f"{name}/populations": ref.populations(), f"{name}/rho": rho, f"{name}/ux": ux,
           f"{name}/uy": uy, f"{name}/uz": uz, f"{name}/force": ref.force(),
           f"{name}/mass": np.array([ref.mass()]), f"{name}/link_cell": cell, f"{name}/link_dir": d,
           f"{name}/link_q": q}
    ref.close()
    return out


def run2d(name: str, steps: int, cfg, mask, init=None) -> dict:
    ref = O.Reference2D(cfg, mask.solid)
    if init is not None:
        ref.initialize(*init)
    ref.step(steps)
    rho, ux, uy = ref.macroscopic()
    out = {f"{name}/populations": ref.populations(), f"{name}/rho": rho, f"{name}/ux": ux,
           f"{name}/uy": uy, f"{name}/force": ref.force(), f"{name}/mass": np.array([ref.mass()])}
    ref.close()
    return out


def main() -> int:
    if not O.reference_available():
        O.build()
    if not O.reference_available():
        print("oracle/_ref is not built (the reference sources are needed)", file=sys.stderr)
        return 1
    O.reference_lib().ref_set_threads(4)
    arrays = {}
    for name, steps, (cfg, mask, init, inlet) in cases.lattice3d_cases():
        arrays.update(run3d(name, steps, cfg, mask, init, inlet))
    for name, steps, (cfg, mask, init) in cases.lattice2d_cases():
        arrays.update(run2d(name, steps, cfg, mask, init))
    # The reference's mask builders.
    for name, (nx, ny, nz, centre, radius) in cases.sphere_masks().items():
        solid, dist = O.reference_sphere_mask(nx, ny, nz, centre, radius)
        arrays[f"mask/{name}/solid"] = solid
        arrays[f"mask/{name}/distance"] = dist
    for name, (nx, ny, nz, lo, hi) in cases.box_masks().items():
        solid, dist = O.reference_box_mask(nx, ny, nz, lo, hi)
        arrays[f"mask/{name}/solid"] = solid
        arrays[f"mask/{name}/distance"] = dist
    for name, (nx, ny, cx, cy, r) in cases.circle_masks().items():
        arrays[f"mask/{name}/solid"] = O.reference_circle_mask(nx, ny, cx, cy, r)
    np.savez_compressed(os.path.join(HERE, "reference_runs.npz"), **arrays)
    # Refusal messages of validate().
    messages = []
    for label, cfg, mask in cases.validation_cases3d():
        messages.append({"label": label, "dims": 3,
                         "message": O.reference_validate3d(cfg, mask.solid, mask.distance)})
    for label, cfg, mask in cases.validation_cases2d():
        messages.append({"label": label, "dims": 2, "message": O.reference_validate2d(cfg, mask.solid)})
    with open(os.path.join(HERE, "validation_messages.json"), "w") as fh:
        json.dump(messages, fh, indent=1)
    print(f"wrote {len(arrays)} arrays and {len(messages)} messages")
    return 0


if __name__ == "__main__":
    sys.exit(main())
