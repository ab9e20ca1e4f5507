"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks agree on the slowest rank's time
and the whole-job throughput; under torchrun the reference arm prints on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(torch, dist, 10.0 * (rank + 1), "cpu")   # rank r took 10 (r+1) ms
        q.put((rank, ms, bench.job_throughput(world, 100, ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [20.0, 20.0]
    assert all(abs(o[2] - 2 * 100 / 0.020) < 1e-9 for o in out)   # both replicas' steps over the job time


def test_single_rank_needs_no_process_group():
    import torch

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(torch, None, 12.5, "cpu") == 12.5


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "2", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
