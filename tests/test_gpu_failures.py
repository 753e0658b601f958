"""Failure detection made to fire, without a GPU fault.

* The staged and tiled steps' bounded mbarrier waits: a stall request makes
  one CTA withhold the copies of its first span or tile (a copy that never
  lands); its
  consumers' bounded wait must give up, the launch must end, and every
  read-back must report ORR_ERR_TIMEOUT until initialize, after which the
  solver steps and reads back exactly like a fresh one.
* Divergence of a served solve: the reference warns ``lbm.diverged`` when the
  coefficients stop being finite (src/aero/lbm3d/lbm_aero_solver3d.cpp:585-588).
  A request made unstable on the host (inlet speed 0.4, tau 0.5005, no closure)
  must end failed with that text, while the requests that shared its batch end
  exactly as they do alone.
"""
import time

import numpy as np
import pytest

from orrery_b200 import abi
from orrery_b200 import solver as S
from orrery_b200 import workloads as W
from orrery_b200._native import LbmError
from orrery_b200.lbm3d import Smagorinsky
from orrery_b200.serve import Server

pytestmark = pytest.mark.gpu


def small(seed, nx=64, ny=32, nz=32, reynolds=60.0):
    return W.sphere3d(seed=seed, nx=nx, ny=ny, nz=nz, diameter=8.0, reynolds=reynolds)


@pytest.mark.parametrize("kernel", ["staged", "tiled"])
def test_staged_wait_runs_out_and_is_reported(kernel):
    w = small(81)
    s = S.make_gpu_solver(w.config, w.mask, storage="f16", kernel=kernel)
    assert s.kernel_info()["kernel"] == kernel
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    s.step(4)
    s.force()
    s.request_stall(0)
    t0 = time.perf_counter()
    s.step(1)
    with pytest.raises(LbmError) as e:
        s.force()
    elapsed = time.perf_counter() - t0
    assert e.value.status == abi.ORR_ERR_TIMEOUT, str(e.value)
    assert elapsed < 30.0
    print(f"stalled launch ended after {elapsed:.2f} s")
    # The populations stay invalid until initialize.
    with pytest.raises(LbmError) as e:
        s.macroscopic()
    assert e.value.status == abi.ORR_ERR_TIMEOUT
    with pytest.raises(LbmError):
        s.populations()
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    s.step(6)
    fresh = S.make_gpu_solver(w.config, w.mask, storage="f16", kernel=kernel)
    fresh.initialize(w.rho, w.ux, w.uy, w.uz)
    fresh.step(6)
    assert np.array_equal(s.populations(), fresh.populations())
    # (the binary64 link sum adds with atomics: equal to its last bits' order)
    fa, fb = s.force().force, fresh.force().force
    assert np.allclose(fa, fb, rtol=0, atol=1e-12 * np.max(np.abs(fb)))
    # Requests the step cannot take are refused.
    with pytest.raises(LbmError):
        s.request_stall(1 << 30)
    rows = S.make_gpu_solver(w.config, w.mask, storage="f32", kernel="rows")
    with pytest.raises(LbmError):
        rows.request_stall(0)
    for h in (s, fresh, rows):
        h.close()


def unstable(seed):
    w = small(seed)
    w.config.inlet_ux = 0.4
    w.config.tau = 0.5005
    w.config.smagorinsky = Smagorinsky(False, 0.0)
    w.allow_high_mach = True
    w.rho = w.ux = w.uy = w.uz = None   # start from the uniform inlet state
    return w


def serve(workloads, delays=None):
    with Server(storage="f32", chunk_steps=100, sample_every=10) as srv:
        ids = []
        for k, w in enumerate(workloads):
            if delays is not None:
                time.sleep(delays[k])
            ids.append(srv.submit(w, window=200, tolerance=2e-3, max_steps=2000))
        srv.drain(timeout=600)
        return [srv.poll(i) for i in ids], srv.stats()


def test_diverging_request_fails_alone_in_its_mix():
    a, b = small(71), small(72, nx=80, ny=32, nz=48, reynolds=100.0)
    bad = unstable(73)
    alone_a, _ = serve([a])
    alone_b, _ = serve([b])
    mixed, stats = serve([a, bad, b], delays=[0.0, 0.02, 0.02])
    r = mixed[1]
    assert r["state"] == "failed", r
    assert "lbm.diverged" in r["message"] and "no longer finite" in r["message"], r["message"]
    assert r["steps"] <= 2000
    for got, want in ((mixed[0], alone_a[0]), (mixed[2], alone_b[0])):
        assert got["state"] in ("converged", "capped")
        for key in ("state", "steps", "cd", "cl", "cm", "delta_cd", "force", "moment"):
            assert got[key] == want[key], (key, got[key], want[key])
    assert stats["failed"] == 1 and stats["completed"] == 2
