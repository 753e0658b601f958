"""Generates tests/golden/oracle32_sphere3d_256x128x128.npz: the force history
of the 256 x 128 x 128 sphere-channel workload (D 32, u 0.05, Re 200,
Smagorinsky C 0.1, seeded +-1e-3 noise, seed 1) over 1000 steps, sampled every
10 steps, from two CPU solvers:

  f64   the reference's own CpuLbm3D (oracle/_ref, compiled from the
        reference sources);
  b32   the binary32 restatement of the reference's GLSL step
        (oracle/lbm_oracle32.c).

Used by tests/test_gpu_fullsize.py to place the CUDA binary32 form's
instantaneous drag against another binary32 evaluation of the same step.
Needs the reference tree at build time (oracle/_ref).

    python tests/golden/make_oracle32_golden.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from orrery_b200 import workloads as W  # noqa: E402

STEPS = 1000
EVERY = 10


def main() -> int:
    w = W.sphere3d(seed=1)
    O.set_threads(os.cpu_count() or 1)
    ref = O.Reference3D(w.config, w.mask.solid, w.mask.distance)
    ref.initialize(w.rho, w.ux, w.uy, w.uz)
    b32 = O.Restated32(w.config, w.mask.solid, ref.links())
    b32.initialize(w.rho, w.ux, w.uy, w.uz)
    series = {"f64": [], "b32": []}
    t0 = time.time()
    for k in range(STEPS // EVERY):
        ref.step(EVERY)
        b32.step(EVERY)
        series["f64"].append(ref.force())
        series["b32"].append(b32.force())
        if k % 10 == 9:
            print(f"{(k + 1) * EVERY} steps, {time.time() - t0:.0f} s", flush=True)
    q = 0.5 * w.config.inlet_ux ** 2 * w.reference_area
    out = os.path.join(HERE, "oracle32_sphere3d_256x128x128.npz")
    np.savez_compressed(out, steps=np.arange(EVERY, STEPS + 1, EVERY), f64=np.array(series["f64"]),
                        b32=np.array(series["b32"]), q=q)
    f64, b32v = np.array(series["f64"])[:, 0] / q, np.array(series["b32"])[:, 0] / q
    print(f"Cd at {STEPS}: f64 {f64[-1]!r}, b32 {b32v[-1]!r} (rel {abs(b32v[-1] - f64[-1]) / abs(f64[-1]):.2e}); "
          f"window mean f64 {f64[-50:].mean()!r}, b32 {b32v[-50:].mean()!r}")
    print("wrote", out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
