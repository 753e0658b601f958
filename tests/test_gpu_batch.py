"""Batches of D3Q19 solvers (orr_batch3d_*): a member stepped in a batch must
hold exactly the populations it holds when stepped alone, whatever the
schedule (one persistent staged launch over all members, or one row-tile
launch per member), the mix of lattice sizes and features, and the split of
the steps; its fixed-order force sums must be the same alone and in a mix.
"""
import numpy as np
import pytest

from helpers import duct_config, sphere_channel
from orrery_b200 import masks as M
from orrery_b200 import solver as S
from orrery_b200 import workloads as W
from orrery_b200.batch import CudaBatch3D
from orrery_b200.lbm3d import Outlet, Smagorinsky, SolidWall, WallKind, wall

pytestmark = pytest.mark.gpu


def lattices(general=False):
    """Four lattices of different sizes and rules, all with the LES closure.
    The default set has periodic or free-slip sides and halfway walls (every
    schedule takes it); `general` swaps in an interpolated wall and no-slip
    duct walls (row schedules only)."""
    out = []
    cfg, mask = sphere_channel(64, 32, 32, 8.0, 2.5, 0.05, 20.0)
    cfg.smagorinsky = Smagorinsky(True, 0.1)
    out.append((cfg, mask))
    cfg, mask = sphere_channel(272, 12, 10, 6.0, 4.0, 0.05, 30.0)     # spans end inside rows
    cfg.smagorinsky = Smagorinsky(True, 0.1)
    if general:
        cfg.outlet = Outlet.convective
    out.append((cfg, mask))
    cfg, mask = sphere_channel(40, 16, 16, 6.0, 2.5, 0.05, 30.0)      # rows not staged
    cfg.smagorinsky = Smagorinsky(True, 0.1)
    if general:
        cfg.solid_wall = SolidWall.interpolated
    out.append((cfg, mask))
    cfg = duct_config(48, 16, 12, 0.8, 1e-5)                            # periodic x, body force
    if not general:
        cfg.y_low = cfg.y_high = wall(WallKind.periodic)
        cfg.z_low = cfg.z_high = wall(WallKind.periodic)
    cfg.smagorinsky = Smagorinsky(True, 0.1)
    out.append((cfg, M.box_mask(48, 16, 12, (10, 4, 3), (16, 9, 8))))
    return out


def solvers(storage, general=False):
    return [S.make_gpu_solver(c, m, storage=storage) for c, m in lattices(general)]


# (kernel, block, stages, nodes per thread, graph branches)
SCHEDULES = [("staged", 256, 2, 2, 0), ("staged", 256, 3, 1, 0), ("staged", 128, 4, 2, 0),
             ("staged", 256, 2, 2, 64), ("staged", 256, 2, 1, 3), ("rows", 128, 0, 0, 0),
             ("rows", 256, 0, 0, 2), ("rows", 128, 0, 2, 0), ("rows", 64, 0, 2, 64)]


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("schedule", SCHEDULES, ids=lambda s: f"{s[0]}{s[1]}s{s[2]}n{s[3]}b{s[4]}")
def test_members_equal_alone(storage, schedule):
    alone = solvers(storage)
    for s in alone:
        s.step(37)
    members = solvers(storage)
    batch = CudaBatch3D()
    for s in members:
        batch.add(s)
    batch.set_schedule(*schedule)
    batch.step(20)    # graph + single steps
    batch.step(17)    # odd split: the next graph starts on the other buffer
    batch.synchronize()
    for a, b in zip(alone, members):
        assert b.steps() == 37
        assert np.array_equal(a.populations(), b.populations())


@pytest.mark.parametrize("general", [False, True], ids=["halfway", "interpolated"])
def test_sampled_forces_alone_and_in_mix(general):
    """Fixed-order force sums: a lattice alone and in a mix of four agree bit
    for bit (with `general`, one member has an interpolated wall: links with
    q != 1/2)."""
    rows = ("rows", 128, 0, 0, 0)
    mixed = solvers("f32", general)
    batch = CudaBatch3D()
    for s in mixed:
        batch.add(s)
    if general:
        batch.set_schedule(*rows)
    sums_mix = batch.step_sampled(100, 10)
    for k, (c, m) in enumerate(lattices(general)):
        solo = S.make_gpu_solver(c, m, storage="f32")
        b1 = CudaBatch3D()
        b1.add(solo)
        if general:
            b1.set_schedule(*rows)
        sums_solo = b1.step_sampled(100, 10)
        assert np.array_equal(sums_solo[0], sums_mix[k])
        # and the same populations
        assert np.array_equal(solo.populations(), mixed[k].populations())
        # the plain force of the member agrees to its rounding
        f = mixed[k].force()
        g = batch.forces()[k]
        assert np.allclose(np.concatenate([f.force, f.moment]), g, rtol=1e-12,
                           atol=1e-12 * np.max(np.abs(g)))


def test_tuner_steps_are_real_steps():
    alone = solvers("f16")
    members = solvers("f16")
    batch = CudaBatch3D()
    for s in members:
        batch.add(s)
    trials = batch.tune(1)
    assert len(trials) >= 4
    assert all(t["ms_per_step"] > 0 for t in trials)
    taken = members[0].steps()
    assert taken > 0 and all(s.steps() == taken for s in members)
    batch.step(10)
    for s in alone:
        s.step(taken + 10)
    for a, b in zip(alone, members):
        assert np.array_equal(a.populations(), b.populations())
    best = min(trials, key=lambda t: t["ms_per_step"])
    sched = batch.schedule()
    assert (sched["kernel"], sched["block"]) == (best["kernel"], best["block"])


def test_membership_rules():
    members = solvers("f32")
    batch = CudaBatch3D()
    batch.add(members[0])
    with pytest.raises(S.LbmError):
        members[0].step(1)            # a member is stepped by its batch
    with pytest.raises(S.LbmError):
        batch.add(members[0])         # already a member
    other = S.make_gpu_solver(*lattices()[0], storage="f16")
    with pytest.raises(S.LbmError):
        batch.add(other)              # another storage form
    plain = S.make_gpu_solver(*lattices()[0], storage="f32")
    batch.add(members[1])
    batch.step(5)
    batch.remove(members[0])
    members[0].step(3)                # its own again
    plain.step(8)
    assert np.array_equal(plain.populations(), members[0].populations())
    members[1].close()                # destroying a member leaves the batch consistent
    batch.members.remove(members[1])
    batch.add(members[2])
    batch.step(4)
    assert batch.size()[0] == 1


def test_reinitialised_member():
    cfg, mask = lattices()[0]
    a = S.make_gpu_solver(cfg, mask)
    b = S.make_gpu_solver(cfg, mask)
    batch = CudaBatch3D()
    batch.add(b)
    batch.step(9)
    w = W.noisy_state3d(cfg, mask, seed=3)
    b.initialize(*w)
    batch.step(6)
    a.initialize(*w)
    a.step(6)
    assert np.array_equal(a.populations(), b.populations())


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_general_members_take_row_schedules(storage):
    """Members with an interpolated wall or no-slip walls next to flat ones:
    row schedules step them exactly as alone; the staged ones are refused."""
    alone = solvers(storage, general=True)
    for s in alone:
        s.step(24)
    members = solvers(storage, general=True)
    batch = CudaBatch3D()
    for s in members:
        batch.add(s)
    batch.set_schedule("staged", 256, 2, 1, 0)
    with pytest.raises(S.LbmError):
        batch.step(2)
    # the pair step on the members it serves (2-byte storage, flat, even nx),
    # the one-node step on the others
    batch.set_schedule("rows", 128, 0, 2, 3)
    batch.step(24)
    for a, b in zip(alone, members):
        assert np.array_equal(a.populations(), b.populations())
    trials = batch.tune(1)
    assert all(t["kernel"] == "rows" for t in trials)
