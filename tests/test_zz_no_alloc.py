"""orr_lbm3d_force_static, the force and moment without device allocation.

Some callers of this library may not allocate device memory (their device
memory belongs to another allocator or pool, or they run a loop that must not
enter the allocator).  orr_lbm3d_force_static serves them with a fixed
scratch array compiled into the library.  This test gives it populations and
link tables that the test itself placed on the device, and checks its result
against orr_lbm3d_force on the same state, twice in a row (the second call
reuses the scratch the first one left behind), for every storage form and
for halfway and interpolated walls, and that a link outside the lattice is
refused.  Collected last so that a failure here does not stop the rest of a
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


def stored_values(f, storage):
    """The device form of read-back populations: f itself for binary64, the
    shifted f - w rounded back to the storage type otherwise (the read-back
    added w in binary64, so rounding recovers the stored value exactly)."""
    import torch
    if storage == "f64":
        return torch.tensor(f.reshape(-1), dtype=torch.float64, device="cuda")
    shifted = torch.tensor((f - W19[:, None]).reshape(-1), dtype=torch.float64, device="cuda")
    return shifted.to({"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[storage])


@pytest.mark.gpu
@pytest.mark.parametrize("storage,wall", [("f64", "halfway"), ("f32", "halfway"), ("f16", "halfway"),
                                          ("bf16", "halfway"), ("f64", "interpolated"),
                                          ("f32", "interpolated"), ("f16", "interpolated")])
def test_force_static_equals_force_on_two_calls_in_a_row(storage, wall):
    import torch
    from orrery_b200.lbm3d import SolidWall
    w = W.sphere3d(seed=4, nx=96, ny=48, nz=48, diameter=12.0)
    if wall == "interpolated":
        w.config.solid_wall = SolidWall.interpolated
    s = S.make_gpu_solver(w.config, w.mask, storage=storage)
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    s.step(200)
    expected = s.force()
    f = s.populations().reshape(19, -1)
    values = stored_values(f, storage)
    cell, direction, q = s.links()
    if wall == "interpolated":
        assert np.any(q < 0.5) and np.any(q > 0.5)
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


@pytest.mark.gpu
def test_force_static_refuses_links_outside_the_lattice():
    """A caller's link whose cell lies beyond the lattice is skipped on the
    device (never read through) and the call is refused; a valid call right
    after it gives the valid result."""
    import torch
    w = W.sphere3d(seed=5, nx=64, ny=32, nz=32, diameter=8.0)
    s = S.make_gpu_solver(w.config, w.mask, storage="f32")
    s.initialize(w.rho, w.ux, w.uy, w.uz)
    s.step(20)
    expected = s.force()
    values = stored_values(s.populations().reshape(19, -1), "f32")
    cell, direction, q = s.links()
    bad_cell = cell.astype(np.int64).copy()
    bad_cell[len(bad_cell) // 2] = w.config.cells + 5
    for cells, dirs, ok in ((bad_cell, direction, False), (cell, direction, True)):
        cell_d = torch.tensor(cells.astype(np.int32), device="cuda")
        dir_d = torch.tensor(dirs.astype(np.int32), device="cuda")
        q_d = torch.tensor(q, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        args = abi.CForceLinks(nx=w.config.nx, ny=w.config.ny, nz=w.config.nz, storage=abi.ORR_STORAGE_F32,
                               device=0, populations=values.data_ptr(), link_cell=cell_d.data_ptr(),
                               link_dir=dir_d.data_ptr(), link_q=q_d.data_ptr(), links=len(cells), stream=None)
        status, out = call_static(args)
        if ok:
            assert status == abi.ORR_OK
            assert np.allclose(out[:3], expected.force, rtol=0, atol=1e-12)
        else:
            assert status == abi.ORR_ERR_INVALID
            assert b"outside the lattice" in _native.lib().orr_last_error()
    s.close()
