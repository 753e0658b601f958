"""Measurement of the batched and served forms of the D3Q19 path.

batched   the 64 NACA-wing lattices of ``workloads.naca_batch`` advanced as
          one batch (``batch.CudaBatch3D``) for a fixed number of steps with
          the force sampled every 10 steps; the schedule is picked by the
          batch autotuner first.  Reported: aggregate MLUPS and solves/s (a
          solve = one lattice for the full step count), next to the plain
          form: the same lattices solved one after another by single binary32
          solvers with the same sampling.
voxelize  the solid mask and wall distances of the largest served body (a
          sphere-cone of 49 K triangles in a 320 x 160 x 160 grid) by
          geometry.voxelize + signed_distance_band on the device.
serve     the sphere-cone request stream of ``workloads.sphere_cone_requests``
          submitted at its (seeded Poisson) arrival times to a ``serve.Server``;
          every solve runs until its window-mean Cd settles or its step cap.
          Reported: solves/s, p50 / p99 latency from arrival to result, and
          the plain form (binary32, one slot: the same requests one after
          another), optionally the Cd error of the first requests (or of every
          converged solve) against the binary64 form of the same solves.

Both return plain dictionaries (bench.py prints them as its JSON line).
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import solver as S
from . import workloads as W
from .batch import CudaBatch3D
from .serve import Server

BYTES_PER_UPDATE = {"f32": 152, "f16": 76, "bf16": 76, "f64": 304}


def run_batched(storage: str = "f32", count: int = 64, steps: int = 3000, seed: int = 4,
                sample_every: int = 10, tune: bool = True, plain: bool = True, warmup: int = 20,
                schedule=None) -> dict:
    import torch

    members = W.naca_batch(seed=seed, count=count)
    total = int(sum(m.cells for m in members))
    # Each lattice is built, uploaded and initialised, and its host arrays
    # dropped, so host memory holds one lattice at a time.
    t0 = time.perf_counter()
    solvers, refs = [], []
    for m in members:
        w = m.build()
        s = S.make_gpu_solver(w.config, w.mask, storage=storage)
        s.initialize(w.rho, w.ux, w.uy, w.uz)
        solvers.append(s)
        refs.append((w.config.inlet_ux, w.reference_area))
        del w
    t_setup = time.perf_counter() - t0
    batch = CudaBatch3D()
    for s in solvers:
        batch.add(s)
    trials = []
    if schedule is not None:
        batch.set_schedule(*schedule)
    elif tune:
        trials = batch.tune(2)
    batch.step(max(warmup, 2) // 2 * 2)
    batch.synchronize()
    # Timed: `steps` steps of every lattice with the force sampled every 10.
    stream = torch.cuda.ExternalStream(batch.stream())
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    launches0 = batch.launch_count()
    start.record(stream)
    t_wall = time.perf_counter()
    sums = batch.step_sampled(steps, sample_every)
    stop.record(stream)
    stop.synchronize()
    wall = time.perf_counter() - t_wall
    ms = start.elapsed_time(stop)
    launches = batch.launch_count() - launches0
    sched = batch.schedule()
    samples = steps // sample_every
    cds = [float(sums[k][0] / samples / (0.5 * u * u * a)) for k, (u, a) in enumerate(refs)]
    out = {
        "form": "batched", "storage": storage, "lattices": count, "nodes": total, "steps": steps,
        "mlups": total * steps / (ms * 1e-3) / 1e6, "ms": ms, "wall_s": wall,
        "solves_per_s": count / (ms * 1e-3),
        "gb_per_s": total * steps * BYTES_PER_UPDATE[storage] / (ms * 1e-3) / 1e9,
        "schedule": sched, "tuning": trials, "gpu_launches": launches,
        "setup_s": t_setup, "cd": cds[:8], "finite": bool(np.all(np.isfinite(sums))),
        "sizes": [(m.nx, m.ny, m.nz) for m in members[:4]],
    }
    batch.close()
    for s in solvers:
        s.close()
    if plain:
        # The plain form: each lattice alone, one after another, same sampling.
        t_plain = 0.0
        for m in members:
            w = m.build()
            s = S.make_gpu_solver(w.config, w.mask, storage="f32")
            s.initialize(w.rho, w.ux, w.uy, w.uz)
            s.step(2)
            torch.cuda.synchronize()
            t = time.perf_counter()
            for _ in range(steps // sample_every):
                s.step(sample_every)
                s.force()
            t_plain += time.perf_counter() - t
            s.close()
            del w
        out["plain"] = {"storage": "f32", "seconds": t_plain, "solves_per_s": count / t_plain,
                        "mlups": total * steps / t_plain / 1e6}
        out["speedup_vs_plain"] = out["solves_per_s"] / out["plain"]["solves_per_s"]
    return out


def _serve_once(requests, workloads, storage, max_active, memory_budget, window, tolerance, max_steps,
                chunk_steps, kernel="auto", branches=0) -> dict:
    with Server(storage=storage, memory_budget=memory_budget, max_active=max_active,
                chunk_steps=chunk_steps, sample_every=10, kernel=kernel, branches=branches) as srv:
        ids = []
        t0 = time.perf_counter()
        caps = max_steps if isinstance(max_steps, (list, tuple)) else [max_steps] * len(requests)
        for r, w, cap in zip(requests, workloads, caps):
            delay = r.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(w, window=window, tolerance=tolerance, max_steps=cap,
                                  initial_state=False))
        srv.drain(timeout=7200)
        results = [srv.poll(i) for i in ids]
        stats = srv.stats()
    states = {}
    for r in results:
        states[r["state"]] = states.get(r["state"], 0) + 1
    return {"storage": storage, "max_active": max_active, "solves_per_s": stats["solves_per_second"],
            "latency_p50_s": stats["latency_p50_s"], "latency_p99_s": stats["latency_p99_s"],
            "latency_mean_s": stats["latency_mean_s"], "completed": stats["completed"],
            "failed": stats["failed"], "states": states, "mean_active": stats["mean_active"],
            "peak_device_gb": stats["peak_device_bytes"] / 1e9,
            "mlups": stats["lattice_updates"] / max(stats["busy_seconds"], 1e-9) / 1e6,
            "steps": [r["steps"] for r in results], "cd": [r["cd"] for r in results],
            "state": [r["state"] for r in results], "worker_message": stats["message"]}


def run_serve(storage: str = "f16", count: int = 48, rate: float = 20.0, seed: int = 5,
              window: int = 500, tolerance: float = 1e-4, max_steps: int = 20000,
              memory_budget: float = 150e9, max_active: int = 64, chunk_steps: int = 100,
              plain: bool = True, oracle_check=0, kernel: str = "auto", branches: int = 0) -> dict:
    requests = W.sphere_cone_requests(seed=seed, count=count, rate=rate)
    t0 = time.perf_counter()
    workloads = []
    for r in requests:
        w = r.build()
        # Halfway walls need no distances; the requests start from the
        # uniform inlet state, so no initial fields either.
        w.mask.distance = None
        w.rho = w.ux = w.uy = w.uz = None
        workloads.append(w)
    t_build = time.perf_counter() - t0
    out = {"form": "serve", "requests": count, "rate_per_s": rate, "window": window,
           "tolerance": tolerance, "max_steps": max_steps, "memory_budget_gb": memory_budget / 1e9,
           "nodes_total": int(sum(r.cells for r in requests)), "host_build_s": t_build}
    out["served"] = _serve_once(requests, workloads, storage, max_active, memory_budget, window, tolerance,
                                max_steps, chunk_steps, kernel, branches)
    out["served"]["schedule"] = {"kernel": kernel, "branches": branches}
    if plain:
        # one slot, binary32, on the row kernel (the single solver's choice
        # for binary32 storage)
        out["plain"] = _serve_once(requests, workloads, "f32", 1, memory_budget, window, tolerance,
                                   max_steps, chunk_steps, "rows", 0)
        out["speedup_vs_plain"] = out["served"]["solves_per_s"] / max(out["plain"]["solves_per_s"], 1e-12)
    if oracle_check == "converged" or (isinstance(oracle_check, int) and oracle_check > 0):
        # Cd against the binary64 form of the same solves at the same step:
        # each binary64 solve is capped at the step its served solve ended
        # on, with a tolerance that never stops it, so both window means
        # cover the same steps.  "converged": every solve that converged;
        # n > 0: the first n requests.
        if oracle_check == "converged":
            pick = [k for k, st in enumerate(out["served"]["state"]) if st == "converged"]
        else:
            pick = list(range(min(oracle_check, count)))
        out["cd_rel_error_vs_f64"] = oracle_errors(out["served"], [requests[k] for k in pick],
                                                   [workloads[k] for k in pick], pick, max_active,
                                                   memory_budget, window, chunk_steps)
    return out


def oracle_errors(served: dict, requests, workloads, pick, max_active, memory_budget, window,
                  chunk_steps) -> dict:
    """Relative Cd error of the served solves `pick` against binary64 solves
    of the same requests capped at the same steps."""
    if not pick:
        return {"n": 0, "max": None, "mean": None, "per_request": [], "requests": [], "steps": [],
                "steps_f64": [], "cd_f64": []}
    caps = [served["steps"][k] for k in pick]
    ref = _serve_once(requests, workloads, "f64", max_active, memory_budget, window, 1e-300, caps,
                      chunk_steps)

    def rel(a, b):
        return abs(a - b) / abs(b) if b else math.inf

    errs = [rel(served["cd"][k], ref["cd"][j]) for j, k in enumerate(pick)]
    out = {"n": len(pick), "max": max(errs), "mean": float(np.mean(errs)), "requests": pick,
           "per_request": errs, "steps": caps, "steps_f64": ref["steps"], "cd_f64": ref["cd"]}
    if served.get("storage") != "f32":
        # The binary32 form of the same solves over the same steps: where the
        # served storage's error matches binary32's, the spread is the
        # trajectories of an unsteady wake parting, not the storage's
        # rounding.
        r32 = _serve_once(requests, workloads, "f32", max_active, memory_budget, window, 1e-300, caps,
                          chunk_steps)
        out["f32_per_request"] = [rel(r32["cd"][j], ref["cd"][j]) for j in range(len(pick))]
        out["cd_f32"] = r32["cd"]
    return out


def voxelize_workload():
    """The largest served body: a sphere-cone (base radius ny / 8, half-angle
    25 degrees, nose radius 0.3 of the base radius; 256 vertices per ring,
    49,152 triangles) at x = nx / 4 of a 320 x 160 x 160 grid of unit cells."""
    from . import geometry as G

    nx, ny, nz = 320, 160, 160
    base = ny / 8.0
    mesh = G.sphere_cone_mesh(base, math.radians(25.0), 0.3 * base, around=256, nose_steps=48, cone_steps=48)
    mesh = G.TriangleMesh(mesh.vertices + np.array([nx / 4.0, ny / 2.0, nz / 2.0]), mesh.triangles)
    return mesh, G.GridSpec((0.0, 0.0, 0.0), 1.0, nx, ny, nz)


def run_voxelize(repeats: int = 5) -> dict:
    """Device voxelization of `voxelize_workload`: cells per second for the
    two kernels (device time by CUDA events inside the library) and end to
    end through the C ABI (host mesh in, host flags and distances out: tree
    build, uploads, kernels, read-backs).  The last results are returned
    under "arrays" for a caller's checks."""
    from . import geometry as G

    mesh, spec = voxelize_workload()
    cells = spec.cells()
    vox = G.voxelize(mesh, spec)          # first call: module load and warm-up
    G.signed_distance_band(mesh, vox)
    dev, wall = [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        vox = G.voxelize(mesh, spec, winding=False)
        sdf = G.signed_distance_band(mesh, vox)
        wall.append(time.perf_counter() - t0)
        dev.append((vox.device_ms + sdf.device_ms) * 1e-3)
    return {"form": "voxelize", "grid": [spec.nx, spec.ny, spec.nz], "cells": cells,
            "triangles": int(len(mesh.triangles)), "solid_cells": vox.solid_count(),
            "band_cells": int(np.count_nonzero(sdf.in_band)), "device_s": min(dev),
            "voxelize_ms": vox.device_ms, "distance_ms": sdf.device_ms,
            "device_mcells_per_s": cells / min(dev) / 1e6, "e2e_s": min(wall),
            "e2e_mcells_per_s": cells / min(wall) / 1e6,
            "h2d_bytes": int(mesh.vertices.nbytes + mesh.triangles.nbytes) * 2 + cells,
            "d2h_bytes": cells * (1 + 8 + 1),
            "arrays": {"solid": vox.solid, "distance": sdf.distance, "in_band": sdf.in_band}}
