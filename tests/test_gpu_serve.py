"""Serving of drag solves with continuous batching (orr_serve_*).

A solve's result must be the same served alone and served in a mix of
requests that arrive while it runs (bit for bit: members of a batch do not
interact and the force sums have a fixed order), the convergence rule must
be the window-mean rule the reference adapter's sampling gives, admission
must respect the device-memory budget, and bad requests are refused.
"""
import time

import numpy as np
import pytest

from orrery_b200 import solver as S
from orrery_b200 import workloads as W
from orrery_b200.lbm3d import XBoundary
from orrery_b200.serve import STEADY_RANGE, Server

pytestmark = pytest.mark.gpu

CHUNK = 100
WINDOW = 200
TOL = 2e-3
CAP = 3000


def small(seed, nx=64, ny=32, nz=32, reynolds=60.0, diameter=8.0):
    return W.sphere3d(seed=seed, nx=nx, ny=ny, nz=nz, diameter=diameter, reynolds=reynolds)


def serve(workloads, storage="f32", delays=None, steady_range=0.0, **opts):
    with Server(storage=storage, chunk_steps=CHUNK, sample_every=10, **opts) as srv:
        ids = []
        for k, w in enumerate(workloads):
            if delays is not None:
                time.sleep(delays[k])
            ids.append(srv.submit(w, window=WINDOW, tolerance=TOL, max_steps=CAP, steady_range=steady_range))
        srv.drain(timeout=600)
        return [srv.poll(i) for i in ids], srv.stats()


def test_results_alone_and_in_mix_are_identical():
    target = small(7)
    alone, _ = serve([target])
    others = [small(11, nx=96, ny=40, nz=40, reynolds=80.0), small(12, nx=48, ny=24, nz=24),
              small(13, nx=80, ny=32, nz=48, reynolds=100.0)]
    # The target arrives between the others, some while they already run.
    mixed, stats = serve([others[0], others[1], target, others[2]], delays=[0.0, 0.0, 0.05, 0.02])
    a, b = alone[0], mixed[2]
    assert a["state"] in ("converged", "capped")
    for key in ("state", "steps", "cd", "cl", "cm", "delta_cd"):
        assert a[key] == b[key], (key, a[key], b[key])
    assert a["force"] == b["force"] and a["moment"] == b["moment"]
    assert stats["completed"] == 4 and stats["failed"] == 0
    assert stats["mean_active"] > 1.0          # the requests overlapped on the device
    assert 0 < stats["latency_p50_s"] <= stats["latency_p99_s"]
    assert stats["solves_per_second"] > 0


@pytest.mark.parametrize("steady_range", [0.0, STEADY_RANGE, 1e-9])
def test_window_rule_matches_a_plain_solver_loop(steady_range):
    """The served steps and window-mean Cd follow the rule run by hand on a
    plain solver (force every 10 steps, window means, |delta Cd| < tol and,
    with a steady range, every force range of the window within that
    fraction of the mean drag force, the reference adapter's steady test).
    A range of 1e-9 holds no window of this flow steady, so that solve runs
    to the cap."""
    w = small(21)
    served, _ = serve([w], steady_range=steady_range)
    r = served[0]
    s = S.make_gpu_solver(w.config, w.mask)
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    q = 0.5 * w.config.inlet_ux ** 2 * w.reference_area
    steps, prev, cd, state = 0, None, None, None
    while state is None:
        samples = []
        for _ in range(WINDOW // 10):
            s.step(10)
            f = s.force()
            samples.append(np.concatenate([f.force, f.moment]))
        samples = np.array(samples)
        acc = np.zeros(6)
        for v in samples:
            acc += v
        steps += WINDOW
        cd = acc[0] / (WINDOW // 10) / q
        mean_fx = acc[0] / (WINDOW // 10)
        ranges = samples[:, :3].max(axis=0) - samples[:, :3].min(axis=0)
        steady = steady_range == 0.0 or bool(np.all(ranges <= steady_range * abs(mean_fx)))
        if prev is not None and abs(cd - prev) < TOL and steady:
            state = "converged"
        elif steps >= CAP:
            state = "capped"
        prev = cd
    s.close()
    assert r["state"] == state
    assert r["steps"] == steps
    assert r["cd"] == pytest.approx(cd, rel=1e-10)
    if steady_range == 1e-9:
        assert state == "capped"


def test_memory_budget_admission():
    ws = [small(31), small(32), small(33)]
    need = max(S.memory_bytes(w.config, 40000, 0, "f32") for w in ws)
    # Room for one lattice at a time.
    results, stats = serve(ws, memory_budget=int(need * 1.5))
    assert all(r["state"] in ("converged", "capped") for r in results)
    assert stats["peak_device_bytes"] <= int(need * 1.5)
    assert stats["mean_active"] == pytest.approx(1.0)
    # Admitted one after another: each starts after the previous finished.
    assert results[1]["admitted_s"] >= results[0]["finished_s"] - 1e-3
    big = small(34, nx=128, ny=64, nz=64)
    res, _ = serve([big], memory_budget=int(need * 1.5))
    assert res[0]["state"] == "failed" and "budget" in res[0]["message"]


def test_served_16bit_and_binary32_within_bar_of_binary64():
    """Cd of a converged served solve in binary16 and binary32 storage against
    the binary64 form of the same request capped at the same step (so both
    window means cover the same steps): within 0.5% relative, always
    asserted."""
    w = small(41)
    for storage in ("f16", "f32"):
        r, _ = serve([w], storage=storage)
        r = r[0]
        assert r["state"] in ("converged", "capped"), (storage, r["state"], r["message"])
        with Server(storage="f64", chunk_steps=CHUNK, sample_every=10) as srv:
            i = srv.submit(w, window=WINDOW, tolerance=1e-300, max_steps=r["steps"])
            srv.drain(timeout=600)
            r64 = srv.poll(i)
        assert r64["steps"] == r["steps"]
        err = abs(r["cd"] - r64["cd"]) / abs(r64["cd"])
        assert err <= 5e-3, (storage, r["cd"], r64["cd"], err)


def test_refusals():
    w = small(51)
    with Server(chunk_steps=CHUNK, sample_every=10) as srv:
        with pytest.raises(S.LbmError):
            srv.submit(w, window=150)            # not a multiple of the chunk
        with pytest.raises(S.LbmError):
            srv.submit(w, tolerance=0.0)
        bad = small(52)
        bad.config.x_boundary = XBoundary.periodic
        with pytest.raises(S.LbmError):
            srv.submit(bad)
    with pytest.raises(S.LbmError):
        Server(chunk_steps=105, sample_every=10)
