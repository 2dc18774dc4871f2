"""The replica path of bench.py with two gloo ranks on the CPU: the
whole-job rate is all ranks' rays over the slowest rank's time, the
collectives run on every rank, and the reference arm does its work on
rank 0 only."""

import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    import bench
    rays = [1000.0, 3000.0][rank]
    ms = [10.0, 20.0][rank]
    rate, ms_max, rays_all = bench.job_rate(rays, ms, world)
    bench.barrier()
    q.put((rank, rate, ms_max, rays_all))
    dist.destroy_process_group()


def _ref_worker(rank, world, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup, blas = 1, 0, 0
    # rank 1 must return before touching the CPU reference or any scene
    out = bench.run_reference(A) if rank != 0 else "skipped"
    q.put((rank, out))


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_job_rate_is_sum_over_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in (0, 1)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, ms_max, rays_all in res:
        assert ms_max == 20.0 and rays_all == 4000.0
        assert rate == pytest.approx(200.0)


def test_reference_arm_runs_on_rank_zero_only():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_worker, args=(1, 2, q))
    p.start()
    rank, out = q.get(timeout=120)
    p.join(timeout=60)
    assert p.exitcode == 0 and rank == 1 and out is None
