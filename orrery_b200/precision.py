"""Precision study: the storage forms of one lattice against its binary64 run.

Runs the same workload with binary64 populations (the FP64 device oracle,
which equals the reference CPU solver bit for bit) and with the binary32,
binary16 and bfloat16 storage forms, sampling the force every `sample_every`
steps like the reference adapter (lbm_aero_solver3d.cpp:385-441).  Reports
per form: Cd, Cl and Cm as window means over the last `window` steps, their
errors relative to the binary64 run, the relative L2 error of the final
velocity field over fluid nodes, and the MLUPS of the form.

    python -m orrery_b200.precision [--workload ellipsoid|sphere] [--scale 1.0]
        [--steps 10000] [--window 2000] [--out results.json]
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import solver as S
from . import workloads as W


def run_form(w: W.Workload3D, storage: str, steps: int, sample_every: int, window: int):
    s = S.make_gpu_solver(w.config, w.mask, storage=storage, allow_high_mach=w.allow_high_mach)
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    samples = []
    t0 = time.perf_counter()
    for _ in range(steps // sample_every):
        s.step(sample_every)
        f = s.force()
        samples.append(np.concatenate([f.force, f.moment]))
    elapsed = time.perf_counter() - t0
    fields = s.macroscopic()
    s.close()
    samples = np.array(samples)
    n = max(1, window // sample_every)
    centre = _body_centre(w)
    mean = samples[-n:].mean(axis=0)
    c = W.coefficients3d(mean[:3], mean[3:], w.config.inlet_ux, w.reference_area, w.reference_length,
                         centre=centre)
    return {"coefficients": c, "fields": fields, "mlups": w.cells * steps / elapsed / 1e6,
            "seconds": elapsed, "finite": bool(np.all(np.isfinite(samples)))}


def _body_centre(w: W.Workload3D):
    solid = w.mask.solid.reshape(w.config.nz, w.config.ny, w.config.nx)
    z, y, x = np.nonzero(solid)
    return (float(x.mean()), float(y.mean()), float(z.mean())) if x.size else (0.0, 0.0, 0.0)


def velocity_error(a, b, solid) -> float:
    keep = solid == 0
    da = np.concatenate([a.velocity_x[keep], a.velocity_y[keep], a.velocity_z[keep]])
    db = np.concatenate([b.velocity_x[keep], b.velocity_y[keep], b.velocity_z[keep]])
    return float(math.sqrt(np.sum((da - db) ** 2) / np.sum(db * db)))


def study(w: W.Workload3D, steps: int, sample_every: int = 10, window: int = 2000,
          forms=("f64", "f32", "f16", "bf16")) -> dict:
    results = {}
    base = None
    for storage in forms:
        r = run_form(w, storage, steps, sample_every, window)
        if base is None:
            base = r
        entry = {"cd": r["coefficients"]["cd"], "cl": r["coefficients"]["cl"], "cm": r["coefficients"]["cm"],
                 "mlups": r["mlups"], "seconds": r["seconds"], "finite": r["finite"]}
        if r is not base:
            bc = base["coefficients"]
            scale = abs(bc["cd"])
            entry["cd_rel_error"] = abs(r["coefficients"]["cd"] - bc["cd"]) / scale
            entry["cl_error_rel_cd"] = abs(r["coefficients"]["cl"] - bc["cl"]) / scale
            entry["cm_error_rel_cd"] = abs(r["coefficients"]["cm"] - bc["cm"]) / scale
            entry["velocity_l2"] = velocity_error(r["fields"], base["fields"], w.mask.solid)
        results[storage] = entry
    return {"workload": w.name, "nodes": w.cells, "steps": steps, "sample_every": sample_every,
            "window": window, "forms": results}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--workload", default="ellipsoid", choices=["ellipsoid", "sphere"])
    ap.add_argument("--scale", type=float, default=1.0, help="lattice size relative to the full workload")
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--window", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    if args.workload == "ellipsoid":
        nx = int(round(512 * args.scale / 8)) * 8
        w = W.ellipsoid3d(seed=args.seed, nx=nx, ny=nx // 2, nz=nx // 2)
    else:
        nx = int(round(256 * args.scale / 8)) * 8
        w = W.sphere3d(seed=args.seed, nx=nx, ny=nx // 2, nz=nx // 2, diameter=32.0 * args.scale)
    out = study(w, args.steps, window=args.window)
    text = json.dumps(out, indent=1)
    print(text)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
