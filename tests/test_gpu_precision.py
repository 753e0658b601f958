"""Accuracy of the storage forms against the binary64 device form (the FP64
oracle, which equals the reference CPU solver bit for bit).

Workload: the precision form's ellipsoid at half scale, 256 x 128 x 128
(semi-axes 24, 12, 12, 10 degrees about z, u 0.08 with the Mach-guard
opt-in, Smagorinsky C 0.12) at the full-size case's relaxation time
(Re 500 on the major axis L = 48 gives nu 0.00768, tau 0.523, as Re 1000 on
L = 96 does), 6000 steps, force sampled every 10 steps, coefficients as means
over the last 2000 steps (the reference adapter reports window means).

Bars: Cd within 0.5% relative; Cl and Cm within 0.5% of |Cd|.
"""
import pytest

from orrery_b200 import precision as P
from orrery_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 6000
WINDOW = 2000
BAR = 5e-3


@pytest.fixture(scope="module")
def study():
    w = W.ellipsoid3d(seed=3, nx=256, ny=128, nz=128, reynolds=500.0)
    return P.study(w, STEPS, sample_every=10, window=WINDOW, forms=("f64", "f32", "f16", "bf16"))


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_coefficients_within_bar(study, storage):
    r = study["forms"][storage]
    assert r["finite"]
    assert r["cd_rel_error"] <= BAR, r
    assert r["cl_error_rel_cd"] <= BAR, r
    assert r["cm_error_rel_cd"] <= BAR, r
    # The velocity field stays close too (full-size figures: 3.6e-5 for
    # binary32, 2.7e-4 for binary16).
    assert r["velocity_l2"] <= 2e-3, r


def test_bfloat16_error_recorded(study):
    """bfloat16 keeps 8 significant bits of f - w, three fewer than binary16:
    at full size its Cd error is 7.1e-3, above the 0.5% bar, so it is not
    held to it.  It must stay finite and within 2%."""
    r = study["forms"]["bf16"]
    assert r["finite"]
    assert r["cd_rel_error"] <= 2e-2, r
    print(f"bf16: Cd rel. error {r['cd_rel_error']:.2e}, velocity L2 {r['velocity_l2']:.2e}")
