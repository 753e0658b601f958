"""The tiled D3Q19 step (tensor copies of 128-node x R-row tiles into shared
memory) against the row-tile step.

The tiled kernel finishes every node with the span kernel's device code
(staged_node3); only where the 19 plain pulls come from changes, so for
every storage form it must give the row kernel's populations bit for bit.
The cases cover the inlet and the zero-gradient and convective outlets at
the x edges of tiled rows, halfway bounce-back next to staged values,
periodic y, periodic x with a body force, the absorbing layers, a row whose
last tile holds 16 nodes (272 = 2 x 128 + 16), and an interior whose last
tile holds fewer rows than the tile (ny - 2 = 19).
"""
import numpy as np
import pytest

from test_gpu_staged import case, run
from orrery_b200 import solver as S

pytestmark = pytest.mark.gpu

CASES = ["sphere_les", "sponge_periodic_y", "periodic_box_obstacle", "ragged_tile", "odd_rows_convective"]


@pytest.mark.parametrize("storage,block", [("f32", 512), ("f16", 512), ("bf16", 512), ("f16", 256),
                                           ("f64", 256)])
@pytest.mark.parametrize("name", CASES)
def test_tiled_equals_rows_bitwise(name, storage, block):
    cfg, mask = case(name)
    a = run(cfg, mask, storage, "rows")
    b = run(cfg, mask, storage, "tiled", block=block)
    info = b.kernel_info()
    assert info["kernel"] == "tiled" and info["block"] == block
    assert info["staged_items"] > 0
    fa, fb = a.populations(), b.populations()
    assert np.array_equal(fa, fb), f"max diff {np.max(np.abs(fa - fb))}"
    ga, gb = a.force().force, b.force().force
    assert np.allclose(ga, gb, rtol=0, atol=1e-12 * np.max(np.abs(ga)))


@pytest.mark.parametrize("block,stages,npt", [(512, 2, 2), (512, 3, 2), (512, 4, 2), (256, 2, 2), (256, 3, 2),
                                              (256, 2, 1), (256, 4, 1)])
@pytest.mark.parametrize("name", ["ragged_tile", "odd_rows_convective"])
def test_tiled_shapes_agree(name, block, stages, npt):
    """Tiles of 8, 4 and 2 rows (two nodes or one per consumer thread)."""
    cfg, mask = case(name)
    ref = run(cfg, mask, "f16", "rows")
    s = run(cfg, mask, "f16", "tiled", block=block, stages=stages, npt=npt)
    info = s.kernel_info()
    assert (info["block"], info["stages"], info["nodes_per_thread"]) == (block, stages, npt)
    assert np.array_equal(ref.populations(), s.populations())


def test_tiled_refuses_lattices_it_cannot_tile():
    for name in ("unaligned_rows", "interpolated_convective_no_slip"):
        cfg, mask = case(name)
        with pytest.raises(S.LbmError):
            S.make_gpu_solver(cfg, mask, storage="f16", kernel="tiled")
