"""orr_lbm3d_force_static, the force and moment without device allocation.

Some callers of this library may not allocate device memory (their device
memory belongs to another allocator or pool, or they run a loop that must not
enter the allocator).  orr_lbm3d_force_static serves them with a fixed
scratch array compiled into the library.  This test gives it populations and
link tables that the test itself placed on the device, and checks its result
against orr_lbm3d_force on the same state, twice in a row (the second call
reuses the scratch the first one left behind), for binary64 and binary32
storage.  Collected last so that a failure here does not stop the rest of a
run that stops at the first failure.
"""
import ctypes

import numpy as np
import pytest

from orrery_b200 import _native, abi
from orrery_b200 import solver as S
from orrery_b200 import workloads as W

W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
_dp = ctypes.POINTER(ctypes.c_double)


def call_static(args):
    out = np.full(6, np.nan)
    status = _native.lib().orr_lbm3d_force_static(ctypes.byref(args), out.ctypes.data_as(_dp))
    return status, out


def test_refuses_more_links_than_the_scratch_holds():
    args = abi.CForceLinks(nx=8, ny=8, nz=8, storage=abi.ORR_STORAGE_F32, device=0,
                           links=abi.ORR_FORCE_STATIC_MAX_LINKS + 1)
    status, _ = call_static(args)
    assert status == abi.ORR_ERR_INVALID
    assert b"exceed" in _native.lib().orr_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_force_static_equals_force_on_two_calls_in_a_row(storage):
    import torch
    w = W.sphere3d(seed=4, nx=96, ny=48, nz=48, diameter=12.0)
    s = S.make_gpu_solver(w.config, w.mask, storage=storage)
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    s.step(200)
    expected = s.force()
    f = s.populations().reshape(19, -1)
    if storage == "f64":
        values = torch.tensor(f.reshape(-1), dtype=torch.float64, device="cuda")
    else:
        # The binary32 form stores f - w; the read-back added w in binary64.
        values = torch.tensor((f - W19[:, None]).astype(np.float32).reshape(-1), device="cuda")
    cell, direction, q = s.links()
    cell_d = torch.tensor(cell.astype(np.int32), device="cuda")
    dir_d = torch.tensor(direction.astype(np.int32), device="cuda")
    q_d = torch.tensor(q, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    args = abi.CForceLinks(nx=w.config.nx, ny=w.config.ny, nz=w.config.nz, storage=abi.STORAGE_NAMES[storage],
                           device=0, populations=values.data_ptr(), link_cell=cell_d.data_ptr(),
                           link_dir=dir_d.data_ptr(), link_q=q_d.data_ptr(), links=len(cell), stream=None)
    first_status, first = call_static(args)
    second_status, second = call_static(args)
    assert first_status == abi.ORR_OK and second_status == abi.ORR_OK
    # Same per-link values as orr_lbm3d_force, summed in another order.
    for out in (first, second):
        assert np.allclose(out[:3], expected.force, rtol=0, atol=1e-12)
        assert np.allclose(out[3:], expected.moment, rtol=0, atol=1e-10)
    # Fixed-order reduction: the two calls agree bit for bit.
    assert np.array_equal(first, second)
    s.close()
