"""Benchmark of the D3Q19 hot path: MLUPS and the fraction of the HBM roofline.

Workload: the 256 x 128 x 128 sphere channel (D 32 at (64, 64, 64), u 0.05,
Re 200, Smagorinsky C 0.1, zero-gradient outflow, free-slip sides), binary32
shifted populations, seeded +-1e-3 velocity noise.  A step is one fused
collide-stream step over the whole lattice; MLUPS counts every node
(steps * nx * ny * nz / s / 1e6).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {cuda,reference}]
  python bench.py --form batched [--storage f16] [--steps 3000]   (64 NACA lattices, one batch)
  python bench.py --form serve [--storage f16]                     (sphere-cone request stream)

N > 1 runs under torchrun as N independent replicas (one lattice per GPU, no
collective on the data path); the reported value is the whole-job MLUPS over
the slowest rank's device time.  ``--impl reference`` times the reference's own
CPU solver (compiled from its sources into oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_UPDATE = {"f32": 152, "f16": 76, "bf16": 76, "f64": 304}  # 2 * 19 * sizeof(storage)
FALLBACK_HBM_GBS = 6650.0


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def dram_traffic(workload: str, storage: str):
    """Per-launch DRAM bytes (read + write) of the step kernel from the
    committed ncu summaries of this workload (a profiles/step3d_*<workload>.md
    line 'traffic_bytes_per_step <storage> <bytes>')."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", f"step3d_*{workload}.md"))):
        try:
            with open(path) as fh:
                for line in fh:
                    parts = line.split()
                    if len(parts) == 3 and parts[0] == "traffic_bytes_per_step" and parts[1] == storage:
                        return float(parts[2])
        except OSError:
            pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"orr_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.remove(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform's processor string."""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_reference_mlups(workload, seconds: float, threads: int | None = None, use_reference=True):
    """Times a CPU solver of the path on the host cores on a bounded sample of
    the workload: the reference's own CpuLbm3D when built (oracle/_ref), else
    the C restatement.  Returns (mlups, cores, kind, sample-description, steps)."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    if use_reference and O.reference_available():
        O.reference_lib().ref_set_threads(threads)
        solver = O.Reference3D(workload.config, workload.mask.solid, workload.mask.distance)
        kind = "reference"
    else:
        O.restated_lib().lo_set_threads(threads)
        solver = O.Restated3D(workload.config, workload.mask.solid, workload.mask.distance)
        kind = "port"
    solver.initialize(workload.rho, workload.ux, workload.uy, workload.uz)
    solver.step(1)  # warm-up
    steps = 0
    t0 = time.perf_counter()
    while True:
        solver.step(1)
        steps += 1
        elapsed = time.perf_counter() - t0
        if elapsed >= seconds or steps >= 2000:
            break
    mlups = steps * workload.cells / elapsed / 1e6
    sample = (f"{steps} steps of the full {workload.config.nx}x{workload.config.ny}x{workload.config.nz} "
              f"lattice after 1 warm-up step, {elapsed:.1f} s wall, {threads} threads of "
              f"{os.cpu_count()} ({cpu_model()})")
    solver.close()
    return mlups, threads, kind, sample, steps


def slowest_rank(value: float, dist=None, device="cuda") -> float:
    """The largest `value` over all ranks (every rank receives it); the value
    itself without a process group.  Times are taken as the slowest rank's."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, steps: int, ms: float, world: int) -> float:
    """Millions of units all ranks processed per second over `ms`, the slowest
    rank's time (every rank runs the same replica size: weak scaling)."""
    return units_per_rank * steps * world / (ms * 1e-3) / 1e6


def run_reference_arm(args, rank: int):
    from orrery_b200 import workloads as W
    if rank != 0:
        return 0
    w = W.sphere3d(seed=1)
    budget = float(os.environ.get("ORR_REFERENCE_SECONDS", "60"))
    per_step_budget = max(budget / max(args.steps + args.warmup, 1), 0.5)
    mlups, cores, kind, sample, steps = cpu_reference_mlups(w, per_step_budget * args.steps)
    line = {
        "impl": "reference", "metric": "D3Q19 MLUPS", "value": mlups, "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": steps, "warmup": 1, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w.name, "storage": "f64 (reference CPU solver)", "seed": 1},
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": cores, "kind": kind, "sample": sample,
                         "cpu_model": cpu_model(), "nproc": os.cpu_count()},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def voxelize_cpu_baseline(forms, arrays, planes: int = 48) -> dict:
    """The reference's own geom::voxelize + geom::signed_distance_band
    (oracle/_ref, single-threaded as in the reference) on `planes` z-planes
    through the middle of the voxelize workload's grid, and whether its output
    equals the device's on those planes."""
    import numpy as np
    from oracle import oracle as O
    if not O.reference_available():
        return {}
    mesh, spec = forms.voxelize_workload()
    k0 = spec.nz // 2 - planes // 2
    origin = (spec.origin[0], spec.origin[1], spec.origin[2] + k0 * spec.spacing)
    n = (spec.nx, spec.ny, planes)
    t0 = time.perf_counter()
    solid, _ = O.reference_voxelize(mesh.vertices, mesh.triangles, origin, spec.spacing, n)
    dist, inb, _ = O.reference_signed_distance_band(mesh.vertices, mesh.triangles, origin, spec.spacing, n, solid)
    seconds = time.perf_counter() - t0
    lo, hi = k0 * spec.nx * spec.ny, (k0 + planes) * spec.nx * spec.ny
    return {"cpu_baseline": {"value": spec.nx * spec.ny * planes / seconds / 1e6, "unit": "Mcells/s", "cores": 1,
                             "kind": "reference", "seconds": seconds,
                             "sample": f"{planes} z-planes of {spec.nx} x {spec.ny} cells through the body's middle"},
            "cpu_slab_matches_device": bool(np.array_equal(solid, arrays["solid"][lo:hi]) and
                                            np.array_equal(dist, arrays["distance"][lo:hi]) and
                                            np.array_equal(inb, arrays["in_band"][lo:hi]))}


def default_forms(args) -> dict:
    """Reduced batched and served forms for the default line (binary16
    storage against the plain binary32 form), small enough to finish in about
    two minutes together: the first 16 lattices of the 64-lattice NACA
    batch for 1000 steps, and the first 16 requests of the sphere-cone stream
    with a 20,000-step cap, the Cd of every converged served solve checked
    against the binary64 form of the same solve at the same step."""
    from orrery_b200 import forms
    out = {}
    t0 = time.perf_counter()
    b = forms.run_batched(storage="f16", count=16, steps=1000, plain=True, warmup=4)
    out["batched"] = {
        "workload": "naca_batch(seed=4)[:16]: 16 NACA-wing lattices (nx 96..256, ny, nz 96..128), 1000 steps, "
                    "force every 10 steps",
        "storage": "f16", "nodes": b["nodes"], "solves_per_s": b["solves_per_s"], "mlups": b["mlups"],
        "plain_f32_solves_per_s": b["plain"]["solves_per_s"], "plain_f32_mlups": b["plain"]["mlups"],
        "speedup_vs_plain": b["speedup_vs_plain"], "schedule": b["schedule"], "gpu_launches": b["gpu_launches"],
        "finite": b["finite"], "seconds": time.perf_counter() - t0}
    t0 = time.perf_counter()
    r = forms.run_serve(storage="f16", count=16, max_steps=20000, plain=True, oracle_check="converged")
    sv, pl, ce = r["served"], r["plain"], r["cd_rel_error_vs_f64"]
    states = {}
    for st in sv["state"]:
        states[st] = states.get(st, 0) + 1
    out["served"] = {
        "workload": "sphere_cone_requests(seed=5)[:16] at 20 req/s: 64^3..320x160x160, Re 100..2000, window 500, "
                    "|dCd| < 1e-4, cap 20,000 steps, 150 GB budget, 64 slots",
        "storage": "f16", "solves_per_s": sv["solves_per_s"], "latency_p50_s": sv["latency_p50_s"],
        "latency_p99_s": sv["latency_p99_s"], "states": states, "mlups": sv["mlups"],
        "plain_f32_solves_per_s": pl["solves_per_s"], "plain_f32_latency_p99_s": pl["latency_p99_s"],
        "speedup_vs_plain": r["speedup_vs_plain"],
        "cd_rel_error_vs_f64": {"converged_checked": ce["n"], "max": ce["max"], "per_request": ce["per_request"],
                                "requests": ce["requests"], "steps": ce["steps"],
                                "within_0.5pct": all(e <= 5e-3 for e in ce["per_request"]),
                                "f32_per_request": ce.get("f32_per_request", []),
                                "within_0.5pct_or_f32_spread": all(
                                    e <= max(5e-3, 2.0 * e32)
                                    for e, e32 in zip(ce["per_request"], ce.get("f32_per_request", [])))},
        "seconds": time.perf_counter() - t0}
    return out


def reference_benchmarks(local_rank: int) -> list:
    """The reference's own GPU benchmark cases (tests/bench/aero/
    bench_lbm_gpu.cpp: D3Q19 128^3 sphere, D2Q9 2048 x 1024 cylinder, BGK and
    Smagorinsky) on the CUDA solver, binary32 as the reference: 50 warm-up
    steps, then 1000 steps timed like the reference (host clock around
    step(1000) and a drain) and on the device (CUDA events on the solver's
    stream).  Beside each, the reference's published rate on its OpenGL
    backend (RX 9060 XT), for context: other hardware."""
    import numpy as np
    import torch

    from orrery_b200 import solver as S
    from orrery_b200 import workloads as W
    out = []
    for case in W.reference_benchmarks():
        s = S.make_gpu_solver(case.config, case.mask)
        stream = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", local_rank))
        s.step(50)
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        start.record(stream)
        s.step(1000)
        stop.record(stream)
        stop.synchronize()
        wall = time.perf_counter() - t0
        device_s = start.elapsed_time(stop) * 1e-3
        finite = bool(np.isfinite(s.mass()))
        s.close()
        out.append({"case": case.name, "nodes": case.cells, "steps_per_s": 1000.0 / wall,
                    "mlups": case.cells * 1000.0 / wall / 1e6, "device_steps_per_s": 1000.0 / device_s,
                    "device_mlups": case.cells * 1000.0 / device_s / 1e6, "finite": finite,
                    "reference_gl_steps_per_s": case.published_steps_per_s,
                    "vs_reference_gl": 1000.0 / wall / case.published_steps_per_s})
    return out


def run_form(args, rank: int) -> int:
    """The batched and served forms (one GPU; other ranks idle)."""
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(0)
    from orrery_b200 import forms
    clocks = ClockSampler(0)
    clocks.start()
    if args.form == "voxelize":
        r = forms.run_voxelize()
        arrays = r.pop("arrays")
        if not args.no_cpu_baseline:
            r.update(voxelize_cpu_baseline(forms, arrays))
        metric, value, unit = "voxelize + distance band Mcells/s", r["device_mcells_per_s"], "Mcells/s"
        clock_info = clocks.stop()
        line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "form": args.form,
                "config": {"workload": "sphere-cone body, 49 K triangles, 320 x 160 x 160 cells"},
                "e2e": {"value": r["e2e_mcells_per_s"], "unit": "Mcells/s", "h2d_bytes_per_step": r["h2d_bytes"],
                        "d2h_bytes_per_step": r["d2h_bytes"]},
                "cpu_baseline": r.get("cpu_baseline"), "result": r, "clocks": clock_info}
        print(json.dumps(line), flush=True)
        return 0
    if args.form == "batched":
        steps = args.steps if args.steps != 1000 else 3000
        r = forms.run_batched(storage=args.storage, count=args.lattices, steps=steps, plain=not args.no_plain,
                              warmup=max(args.warmup, 4))
        metric, value, unit = "D3Q19 batched solves/s", r["solves_per_s"], "solves/s"
    else:
        r = forms.run_serve(storage=args.storage, count=args.requests, max_steps=args.max_steps,
                            plain=not args.no_plain, oracle_check=args.oracle_check,
                            kernel=args.serve_kernel, branches=args.serve_branches)
        metric, value, unit = "D3Q19 served solves/s", r["served"]["solves_per_s"], "solves/s"
    clock_info = clocks.stop()
    peak, peak_kind = measured_peak()
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "f32", "f16": "f16-storage/f32-math", "bf16": "bf16-storage/f32-math",
                      "f64": "f64"}[args.storage],
            "data": "synthetic", "form": args.form, "result": r, "clocks": clock_info,
            "hbm_peak_gbs": peak, "peak_source": peak_kind}
    print(json.dumps(line), flush=True)
    return 0


def _oracle_check(text: str):
    return text if text == "converged" else int(text)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f64"])
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--kernel", default="auto", choices=["auto", "rows", "staged", "tiled"])
    ap.add_argument("--stages", type=int, default=0)
    ap.add_argument("--npt", type=int, default=0, help="nodes per thread of a staged span, or of the row kernel (2: the pair step)")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "serve", "voxelize"])
    ap.add_argument("--lattices", type=int, default=64, help="batched form: lattices")
    ap.add_argument("--requests", type=int, default=48, help="serve form: requests")
    ap.add_argument("--max-steps", type=int, default=20000, help="serve form: step cap per solve")
    ap.add_argument("--oracle-check", type=_oracle_check, default=0,
                    help="serve form: the first N requests, or 'converged' (every solve that settled), "
                         "whose Cd is checked against the binary64 and binary32 forms")
    ap.add_argument("--no-plain", action="store_true", help="batched/serve: skip the plain-form baseline")
    ap.add_argument("--serve-kernel", default="auto", choices=["auto", "rows", "staged"],
                    help="serve form: the batch schedule's kernel")
    ap.add_argument("--serve-branches", type=int, default=0,
                    help="serve form: parallel graph branches of per-lattice launches (0: one launch / stream)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=1000)
    ap.add_argument("--no-forms", action="store_true",
                    help="plain form: leave out the reduced batched and served forms of the default line")
    ap.add_argument("--e2e-repeats", type=int, default=3,
                    help="whole solves timed end to end; the line reports their median")
    args = ap.parse_args(argv)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    if args.form != "plain":
        return run_form(args, rank)

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    else:
        torch.cuda.set_device(0)

    from orrery_b200 import solver as S
    from orrery_b200 import workloads as W

    w = W.sphere3d(seed=1 + rank)
    solver = S.make_gpu_solver(w.config, w.mask, storage=args.storage, device=local_rank,
                               block_x=args.block, kernel=args.kernel, stages=args.stages,
                               nodes_per_thread=args.npt)
    kinfo = solver.kernel_info()
    solver.initialize(w.rho, w.ux, w.uy, w.uz)
    stream = torch.cuda.ExternalStream(solver.stream(), device=torch.device("cuda", local_rank))
    warmup = max(args.warmup, 3)
    solver.step(warmup)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local_rank) if rank == 0 else None
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    launches_before = solver.launch_count()
    barrier()
    if clocks:
        clocks.start()
    start.record(stream)
    solver.step(args.steps)
    stop.record(stream)
    stop.synchronize()
    barrier()
    clock_info = clocks.stop() if clocks else None
    launches = solver.launch_count() - launches_before
    ms = slowest_rank(start.elapsed_time(stop), dist)
    ms_per_step = ms / args.steps
    mlups = whole_job_rate(w.cells, args.steps, ms, world)

    # Roofline of the step (bulk + boundary kernels): algorithmic bytes per
    # step over the device time of a step.
    bytes_per_step = BYTES_PER_UPDATE[args.storage] * w.cells
    achieved_gbs = bytes_per_step / (ms_per_step * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = dram_traffic(w.name, args.storage)
    solver.close()

    # End to end through the C ABI with host buffers: create from the host
    # mask, initialise from host fields, step with the force read back every
    # 10 steps (the reference adapter's sampling), read the moments back.
    e2e = None
    if args.e2e_steps >= 10 and args.e2e_repeats >= 1:
        import numpy as np
        samples = args.e2e_steps // 10
        times, phases, fx = [], [], []
        for _ in range(args.e2e_repeats):
            barrier()
            t0 = time.perf_counter()
            s2 = S.make_gpu_solver(w.config, w.mask, storage=args.storage, device=local_rank, block_x=args.block,
                                   kernel=args.kernel, stages=args.stages, nodes_per_thread=args.npt)
            t1 = time.perf_counter()
            s2.initialize(w.rho, w.ux, w.uy, w.uz)
            t2 = time.perf_counter()
            fx_run = []
            for _ in range(samples):
                s2.step(10)
                fx_run.append(s2.force().force[0])
            t3 = time.perf_counter()
            fx = fx_run
            fields = s2.macroscopic()
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            times.append(slowest_rank(t4 - t0, dist))
            # this rank's phases (the whole solve above is the slowest rank's)
            phases.append({"create": (t1 - t0) * 1e3, "initialize": (t2 - t1) * 1e3,
                           "steps_and_forces": (t3 - t2) * 1e3, "macroscopic": (t4 - t3) * 1e3})
            del fields
            s2.close()
        e2e_s = float(np.median(times))
        mid = phases[int(np.argsort(times)[len(times) // 2])]
        k = samples * 10
        h2d = w.cells * (1 + 4 * 8) + 8 * 3  # mask, four initial fields, inlet velocity
        d2h = samples * 48 + 4 * 8 * w.cells
        e2e = {"value": w.cells * k * world / e2e_s / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": h2d / k, "d2h_bytes_per_step": d2h / k,
               "steps": k, "seconds": e2e_s, "seconds_each": times,
               "phases_ms": {key: round(v, 2) for key, v in mid.items()},
               "note": f"whole solves per rank, median of {len(times)}: create (plan + upload), initialise from "
                       "host fields, steps with the force read back every 10 steps, moments read back"}
        # The drag coefficient the reference adapter reports: the mean of the
        # last 50 force samples (every 10 steps) over 1/2 rho U^2 A.
        window = fx[-50:]
        u = w.config.inlet_ux
        e2e["cd_window_mean"] = float(np.mean(window)) / (0.5 * u * u * w.reference_area)
        e2e["cd_window"] = (f"mean Fx of the last {len(window)} force samples of the last solve "
                            f"(steps {k - 10 * (len(window) - 1)}..{k}) over 1/2 rho U^2 A, A = pi D^2 / 4; "
                            "impulsive start from noisy uniform flow, so not yet the steady drag")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        secs = float(os.environ.get("ORR_CPU_BASELINE_SECONDS", "30"))
        mlups_cpu, cores, kind, sample, _ = cpu_reference_mlups(w, secs)
        cpu = {"value": mlups_cpu, "unit": "MLUPS", "cores": cores, "kind": kind, "sample": sample,
               "cpu_model": cpu_model(), "nproc": os.cpu_count()}

    forms_out = None
    ref_cases = None
    if rank == 0 and world == 1 and not args.no_forms:
        ref_cases = reference_benchmarks(local_rank)
        forms_out = default_forms(args)

    if rank == 0:
        line = {
            "metric": "D3Q19 MLUPS", "value": mlups, "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "f32", "f16": "f16-storage/f32-math", "bf16": "bf16-storage/f32-math",
                      "f64": "f64"}[args.storage],
            "data": "synthetic",
            "config": {"workload": w.name, "nodes": w.cells, "storage": args.storage,
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": f"inputs larger than L2: {w.cells * 19 * {'f32': 4, 'f16': 2, 'bf16': 2, 'f64': 8}[args.storage] / 1e6:.0f} MB per population buffer",
                       "seed": 1, "kernel": kinfo},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                         "frac": achieved_gbs / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_node": BYTES_PER_UPDATE[args.storage]},
            "gpu_launches": launches,
            "clocks": clock_info,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        if forms_out is not None:
            line["forms"] = forms_out
        if ref_cases is not None:
            line["reference_benchmarks"] = ref_cases
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
