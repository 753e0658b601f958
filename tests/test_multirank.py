"""The multi-rank path of bench.py on CPU (world size 2, gloo).

`bench.py --gpus N` runs one replica per rank with no collective on the data
path (the lattices are independent); the ranks meet only to time the run:
a barrier on both sides, then the largest time over the ranks, from which the
whole-job rate is computed with every rank's work.  These tests run that
reduction over a real two-process gloo group, and check that the reference
arm's other ranks exit without work.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = bench.slowest_rank(times[rank], dist, device="cpu")
        rate = bench.whole_job_rate(4_194_304, 1000, ms, world)
        dist.barrier()
        out.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_the_slowest_and_count_all_work():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    times = [101.5, 104.25]                      # ms of the two replicas
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(out.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [104.25, 104.25]  # every rank reports the slowest time
    expected = 4_194_304 * 1000 * 2 / (104.25e-3) / 1e6
    assert all(abs(g[2] - expected) < 1e-9 * expected for g in got)


def test_single_rank_is_its_own_slowest():
    assert bench.slowest_rank(12.5) == 12.5
    assert bench.whole_job_rate(100, 10, 1.0, 1) == pytest.approx(1.0)


def test_reference_arm_other_ranks_exit_without_work():
    class Args:
        steps = 3
        warmup = 1
        gpus = 2
    assert bench.run_reference_arm(Args(), rank=1) == 0


def test_replicas_are_independent_lattices():
    """Rank r runs the seeded workload with seed 1 + r: same size, own noise."""
    from orrery_b200 import workloads as W
    a, b = W.sphere3d(seed=1, nx=32, ny=16, nz=16, diameter=6.0), W.sphere3d(seed=2, nx=32, ny=16, nz=16,
                                                                              diameter=6.0)
    assert a.cells == b.cells
    assert not (a.ux == b.ux).all()
