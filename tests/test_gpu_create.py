"""Creation of a device solver: the buffers sized by the configuration are
allocated on a helper thread while the host plans the lattice, and the full
memory check (check_memory, lbm3d_gpu.cpp:129-149) follows the plan.  These
cases check that creation and destruction return every byte, and that a
lattice that does not fit is refused with the memory status and text before
anything is allocated."""
import numpy as np
import pytest
import torch

from orrery_b200 import abi
from orrery_b200 import solver as S
from orrery_b200 import workloads as W
from orrery_b200.lbm3d import periodic_box
from orrery_b200.masks import SolidMask3D

pytestmark = pytest.mark.gpu


def _free():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def _cycle(w, storage):
    with S.make_gpu_solver(w.config, w.mask, storage=storage) as s:
        s.initialize(w.rho, w.ux, w.uy, w.uz)
        s.step(2)
        assert np.isfinite(s.force().force).all()
        s.macroscopic()


def test_create_and_close_return_all_device_memory():
    w = W.sphere3d(seed=1, nx=128, ny=64, nz=64, diameter=16.0)
    storages = ("f32", "f16", "bf16", "f64")
    for storage in storages:        # first use: context, each storage's kernels, staging ring
        _cycle(w, storage)
    before = _free()
    for storage in storages + ("f32",):
        _cycle(w, storage)
    assert _free() == before


def test_a_lattice_larger_than_free_memory_is_refused():
    nx, ny, nz = 256, 256, 256                 # 1.3 GB of binary32 populations and tables
    cfg = periodic_box(nx, ny, nz, 0.8)
    mask = SolidMask3D(nx, ny, nz, np.zeros(nx * ny * nz, np.uint8), None)
    assert S.memory_bytes(cfg, 0, 0) > (256 << 20)
    # Hold all but about 256 MiB of the free device memory, a GiB at a time.
    hold = []
    while _free() > (256 << 20) + (1 << 30):
        hold.append(torch.empty(1 << 30, dtype=torch.uint8, device="cuda"))
    hold.append(torch.empty(_free() - (256 << 20), dtype=torch.uint8, device="cuda"))
    try:
        with pytest.raises(S.LbmError) as e:
            S.make_gpu_solver(cfg, mask)
        assert e.value.status == abi.ORR_ERR_MEMORY
        assert "of device memory" in str(e.value) and "are available; use fewer cells" in str(e.value)
    finally:
        del hold
        torch.cuda.empty_cache()
    # the same lattice fits once the memory is back
    with S.make_gpu_solver(cfg, mask) as s:
        s.step(1)
