"""The persistent staged D3Q19 step against the row-tile step.

Both kernels finish every node with the same device code (the staged kernel
only changes where the 19 plain pulls come from: a shared-memory stage
instead of global loads), so for every storage form they must give the same
populations bit for bit.  The cases cover each rule the staged kernel has to
route correctly: the inlet and the zero-gradient outlet at the x edges of
interior rows, halfway bounce-back next to staged values, periodic y and
periodic x with a body force, the absorbing layers, spans that end inside a
row or hold several rows, and lattices whose rows cannot be staged (every row
on the per-node path).  Lattices with no-slip sides or interpolated walls are
refused by the staged kernel.
"""
import numpy as np
import pytest

from helpers import copy_config, duct_config, sphere_channel
from orrery_b200 import masks as M
from orrery_b200 import solver as S
from orrery_b200.lbm3d import Outlet, Smagorinsky, SolidWall, Sponge, WallKind, wall

pytestmark = pytest.mark.gpu

STEPS = 150


def case(name):
    if name == "sphere_les":
        cfg, mask = sphere_channel(64, 32, 32, 8.0, 2.5, 0.05, 20.0)
        cfg.smagorinsky = Smagorinsky(True, 0.1)
        return cfg, mask
    if name == "sponge_periodic_y":
        cfg, mask = sphere_channel(64, 24, 20, 7.0, 3.0, 0.05, 40.0)
        cfg.sponge = Sponge(0.5, 6, 8, 4)
        cfg.y_low = wall(WallKind.periodic)
        cfg.y_high = wall(WallKind.periodic)
        cfg.smagorinsky = Smagorinsky(True, 0.12)
        return cfg, mask
    if name == "periodic_box_obstacle":
        # periodic in all three directions, body force, a box obstacle
        cfg = duct_config(48, 16, 12, 0.8, 1e-5)
        cfg.y_low = cfg.y_high = wall(WallKind.periodic)
        cfg.z_low = cfg.z_high = wall(WallKind.periodic)
        mask = M.box_mask(48, 16, 12, (10, 4, 3), (16, 9, 8))
        return cfg, mask
    if name == "interpolated_convective_no_slip":
        # not staged: the rows kernel must refuse nothing, the staged one refuses
        cfg, mask = sphere_channel(64, 24, 20, 7.0, 3.0, 0.05, 40.0)
        cfg.solid_wall = SolidWall.interpolated
        cfg.outlet = Outlet.convective
        cfg.z_low = wall(WallKind.no_slip, 0.01)
        cfg.z_high = wall(WallKind.no_slip, -0.02)
        return cfg, mask
    if name == "ragged_tile":
        # 272 = 256 + 16: the second tile of a 256-node row holds 16 nodes.
        cfg, mask = sphere_channel(272, 12, 10, 6.0, 4.0, 0.05, 30.0)
        return cfg, mask
    if name == "unaligned_rows":
        # nx = 40 is not a multiple of 16: every row takes the per-node path.
        cfg, mask = sphere_channel(40, 16, 16, 6.0, 2.5, 0.05, 30.0)
        return cfg, mask
    if name == "odd_rows_convective":
        # ny = 21: the last row of a two-row block stands alone; convective outlet.
        cfg, mask = sphere_channel(48, 21, 17, 7.0, 3.0, 0.05, 40.0)
        cfg.outlet = Outlet.convective
        return cfg, mask
    raise KeyError(name)


CASES = ["sphere_les", "sponge_periodic_y", "periodic_box_obstacle", "ragged_tile", "unaligned_rows"]


def run(cfg, mask, storage, kernel, block=0, stages=0, steps=STEPS, inlet=None, npt=0):
    s = S.make_gpu_solver(cfg, mask, storage=storage, kernel=kernel, block_x=block, stages=stages,
                          nodes_per_thread=npt)
    if inlet is not None:
        s.set_inlet_velocity(inlet)
    s.step(steps)
    return s


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("name", CASES)
def test_staged_equals_rows_bitwise(name, storage):
    cfg, mask = case(name)
    a = run(cfg, mask, storage, "rows")
    b = run(cfg, mask, storage, "staged")
    info = b.kernel_info()
    assert info["kernel"] == "staged"
    if name == "unaligned_rows":
        assert info["staged_items"] == 0
    else:
        assert info["staged_items"] > 0
    fa, fb = a.populations(), b.populations()
    assert np.array_equal(fa, fb), f"max diff {np.max(np.abs(fa - fb))}"
    # Equal populations; the binary64 link sum adds with atomics, so only its
    # last bits may depend on the order.
    ga, gb = a.force().force, b.force().force
    assert np.allclose(ga, gb, rtol=0, atol=1e-12 * np.max(np.abs(ga)))


@pytest.mark.parametrize("block,stages,npt", [(128, 1, 1), (128, 3, 2), (256, 2, 1), (256, 4, 1), (256, 2, 2),
                                              (256, 3, 2)])
@pytest.mark.parametrize("name", ["sphere_les", "ragged_tile", "sponge_periodic_y"])
def test_launch_shapes_agree(name, block, stages, npt):
    """Spans of one or two nodes per thread, across rows (64 and 272 nodes
    wide: spans hold several rows, or end inside one)."""
    cfg, mask = case(name)
    ref = run(cfg, mask, "f32", "rows")
    s = run(cfg, mask, "f32", "staged", block=block, stages=stages, npt=npt)
    info = s.kernel_info()
    assert (info["block"], info["stages"], info["nodes_per_thread"]) == (block, stages, npt)
    assert np.array_equal(ref.populations(), s.populations())


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("name", CASES + ["odd_rows_convective"])
def test_pair_step_bitwise(name, storage):
    """The pair step (two neighbouring nodes per thread, packed collision)
    rounds every value as the one-node row step: equal populations bit for
    bit, across tiles that end inside a row and warps past the row end."""
    cfg, mask = case(name)
    a = run(cfg, mask, storage, "rows")
    for block in (128, 64, 32):
        b = run(cfg, mask, storage, "rows", block=block, npt=2)
        info = b.kernel_info()
        assert (info["kernel"], info["nodes_per_thread"], info["block"]) == ("rows", 2, block)
        fa, fb = a.populations(), b.populations()
        assert np.array_equal(fa, fb), f"block {block}: {np.count_nonzero(fa != fb)} values differ"


def test_skewed_inlet_bitwise():
    cfg, mask = case("sphere_les")
    cfg = copy_config(cfg)
    a = run(cfg, mask, "f64", "rows", inlet=(0.04, 0.004, -0.003))
    b = run(cfg, mask, "f64", "staged", inlet=(0.04, 0.004, -0.003))
    assert np.array_equal(a.populations(), b.populations())


def test_automatic_choice():
    """The automatic choice is the row kernel for every storage; the staged
    step runs when asked for."""
    cfg, mask = case("sphere_les")
    for storage in ("f16", "bf16", "f32", "f64"):
        assert S.make_gpu_solver(cfg, mask, storage=storage).kernel_info()["kernel"] == "rows"
    assert S.make_gpu_solver(cfg, mask, storage="f16", kernel="staged").kernel_info()["kernel"] == "staged"
    cfg, mask = case("unaligned_rows")
    assert S.make_gpu_solver(cfg, mask, storage="f16").kernel_info()["kernel"] == "rows"
    cfg, mask = case("sphere_les")
    assert S.make_gpu_solver(cfg, mask, storage="f16", kernel="rows").kernel_info()["kernel"] == "rows"


def test_staged_refuses_general_boundaries():
    cfg, mask = case("interpolated_convective_no_slip")
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, storage="f16", kernel="staged")
    # the automatic choice takes the row kernel for it
    assert S.make_gpu_solver(cfg, mask, storage="f16").kernel_info()["kernel"] == "rows"
    # the pair step: 2-byte storage on flat lattices with even nx only
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, storage="f16", kernel="rows", nodes_per_thread=2)
    cfg, mask = case("sphere_les")
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, storage="f32", kernel="rows", nodes_per_thread=2)
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, storage="f16", kernel="rows", nodes_per_thread=2, block_x=256)
    cfg, mask = sphere_channel(45, 16, 16, 6.0, 2.5, 0.05, 30.0)
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, storage="f16", kernel="rows", nodes_per_thread=2)


def test_refused_shapes():
    cfg, mask = case("sphere_les")
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, kernel="staged", block_x=64)
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, kernel="staged", stages=9)
    with pytest.raises(S.LbmError):
        S.make_gpu_solver(cfg, mask, kernel="staged", nodes_per_thread=3)
