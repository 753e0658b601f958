"""Drag tables on the serving loop: the served counterpart of the reference's
``atmo::sample_cd_table``.

``atmo::sample_cd_table`` (src/atmo/cd_sampling.cpp:98-120) builds a Cd(Mach)
table by running one ``IAeroSolver`` per Mach number, one after another
(``solve``, cd_sampling.cpp:47-56).  With the lattice Boltzmann solver,
``LbmAeroSolver3D`` (src/aero/lbm3d/lbm_aero_solver3d.cpp), every point is one
lattice solve of fixed length: it starts at rest, raises the inlet velocity
over ``ramp_steps`` lattice steps (:398-412), samples the force every
``sample_every`` steps, runs ``total_steps`` steps and reports the
coefficients of the mean force over the last ``window_samples`` samples
(:464-481).

``serve_cd_table`` submits every point's lattice solve to one server at once
in that run mode (``ORR_RUN_FIXED_STEPS`` with the gradual start), so the
points share the device and overlap instead of running one after another,
and assembles what the reference's ``AeroCoefficientTable`` holds: the
samples (Mach, Cd), strictly increasing in Mach, with piecewise-linear
lookup held constant beyond the ends (src/atmo/aero_table.cpp:24-83).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import masks as M
from .lbm3d import Lbm3DConfig
from .serve import Server
from .workloads import Workload3D


@dataclass
class LatticeProblem:
    """One Mach point's lattice solve as LbmAeroSolver3D::setup builds it."""
    mach: float
    config: Lbm3DConfig
    solid: np.ndarray              # nx*ny*nz flags
    distance: np.ndarray | None    # signed wall distances (interpolated wall) or None
    total_steps: int               # lattice steps of the run
    window_samples: int            # force samples in the averaging window
    ramp_steps: float              # lattice steps of the gradual start (0: none)
    area: float                    # reference area, lattice units (A / dx^2)
    length: float                  # reference length, lattice units
    sample_every: int = 10
    allow_high_mach: bool = False

    @property
    def window_steps(self) -> int:
        return self.window_samples * self.sample_every


@dataclass
class CdLookup:
    cd: float
    clamped: bool


class CdTable:
    """Cd against Mach (AeroCoefficientTable, src/atmo/aero_table.cpp:24-83):
    samples strictly increasing in Mach with positive finite Cd; lookup
    interpolates linearly and holds the end values beyond the ends."""

    def __init__(self, samples):
        samples = [(float(m), float(c)) for m, c in samples]
        if not samples:
            raise ValueError("the table needs at least one sample")
        for i, (m, c) in enumerate(samples):
            if not math.isfinite(m) or m < 0.0:
                raise ValueError(f"sample {i}: Mach must be finite and non-negative")
            if not (c > 0.0 and math.isfinite(c)):
                raise ValueError(f"sample {i}: Cd must be positive and finite")
            if i > 0 and not m > samples[i - 1][0]:
                raise ValueError(f"sample {i}: Mach numbers must be strictly increasing")
        self.samples = samples

    def lookup(self, mach: float) -> CdLookup:
        first, last = self.samples[0], self.samples[-1]
        if not mach > first[0]:
            return CdLookup(first[1], mach != first[0])
        if mach >= last[0]:
            return CdLookup(last[1], mach != last[0])
        k = next(i for i, (m, _) in enumerate(self.samples) if mach < m)
        (m0, c0), (m1, c1) = self.samples[k - 1], self.samples[k]
        f = (mach - m0) / (m1 - m0)
        return CdLookup(c0 + f * (c1 - c0), False)

    def cd(self, mach: float) -> float:
        return self.lookup(mach).cd


def serve_cd_table(problems: list[LatticeProblem], storage: str = "f32", memory_budget: float = 150e9,
                   max_active: int = 64, timeout: float = 7200.0) -> dict:
    """Runs every point of a drag table on one server at once and returns
    {"table": CdTable, "points": [per-point result dicts], "stats": ...}.
    Raises ValueError for a point that fails or whose Cd is not positive and
    finite (the reference's sample_point refusal, cd_sampling.cpp:90-94)."""
    if not problems:
        raise ValueError("at least one Mach number is needed")
    every = problems[0].sample_every
    if any(p.sample_every != every for p in problems):
        raise ValueError("every point must sample the force at the same interval")
    # Rounds that end on every point's window start and run end.
    chunk = 0
    for p in problems:
        if p.total_steps % every != 0 or p.total_steps < p.window_steps:
            raise ValueError(f"Mach {p.mach}: the run of {p.total_steps} steps must be a multiple of "
                             f"{every} and hold its window of {p.window_steps} steps")
        chunk = math.gcd(chunk, math.gcd(p.total_steps, p.window_steps))
    with Server(storage=storage, memory_budget=memory_budget, max_active=max_active, chunk_steps=chunk,
                sample_every=every) as srv:
        ids = []
        for p in problems:
            mask = M.SolidMask3D(p.config.nx, p.config.ny, p.config.nz, p.solid, p.distance)
            w = Workload3D(f"mach_{p.mach:g}", p.config, mask, None, None, None, None, p.length, p.area,
                           allow_high_mach=p.allow_high_mach)
            ids.append(srv.submit(w, window=p.window_steps, max_steps=p.total_steps, initial_state=False,
                                  fixed_steps=True, ramp_steps=p.ramp_steps))
        srv.drain(timeout=timeout)
        results = [srv.poll(i) for i in ids]
        stats = srv.stats()
    samples = []
    for p, r in zip(problems, results):
        if r["state"] != "completed":
            raise ValueError(f"Mach {p.mach}: the solve ended {r['state']}: {r['message']}")
        if not (r["cd"] > 0.0 and math.isfinite(r["cd"])):
            raise ValueError(f"Mach {p.mach}: the solver returned Cd {r['cd']}")
        samples.append((p.mach, r["cd"]))
    return {"table": CdTable(samples), "points": results, "stats": stats, "chunk_steps": chunk}
