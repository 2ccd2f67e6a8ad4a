"""bench.py's multi-rank plumbing on CPU: two gloo ranks (the layout that
torchrun gives the GPU runs, with gloo in place of NCCL) agree on the
slowest rank's time, the whole-job value counts every rank's units, and the
reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, REPO)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup("gloo")
    assert (w, r, local) == (world, rank, rank)
    ms_local = 100.0 + 50.0 * rank  # rank 1 is the slower one
    bench.dist_barrier(w)
    ms_max = bench.dist_max(ms_local, w)
    value = bench.whole_job_value(2_000_000, w, ms_max)
    out.put((rank, ms_max, value))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, ms_max, value in got:
        assert ms_max == 150.0
        # 2 ranks x 2 Mpx in 0.15 s of the slowest rank.
        assert value == pytest.approx(2 * 2.0 / 0.15)


def test_single_rank_value():
    sys.path.insert(0, REPO)
    import bench
    assert bench.dist_max(3.5, 1) == 3.5
    assert bench.whole_job_value(1e6, 1, 1000.0) == pytest.approx(1.0)


def _ref_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, REPO)
    import bench

    class Args:
        steps, warmup, frames = 1, 3, 2
    ran = []

    def stop(specs):  # the first thing the reference arm does on its rank
        ran.extend(s["name"] for s in specs)
        raise RuntimeError("stop")
    from rv9 import workloads
    workloads.ensure_cached = stop
    w, r, _ = bench.dist_setup("gloo")
    try:
        bench.run_reference(Args, w, r)
    except RuntimeError:
        pass
    out.put((rank, bool(ran)))
    import torch.distributed as dist
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_reference_arm_runs_on_rank_zero_only():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ref_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=100) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
    assert got == {0: True, 1: False}
