"""The multi-GPU bench path is replicas only: every rank runs the whole scan on its own GPU, and the job's time is the
slowest rank's. These tests run that aggregation as two CPU ranks over gloo (the GPU runs use nccl), and check that the
reference arm's non-zero ranks leave without work or output. CPU only."""

import datetime
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = 100.0 + 50.0 * rank          # the second rank is slower
        slow = bench.slowest_rank(ms, dist, "cpu")
        e2e = bench.slowest_rank(2.0 - rank, dist, "cpu")
        q.put((rank, slow, bench.whole_job_rate(81920, world, slow / 1e3), e2e))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank, slow, rate, e2e in results:
        assert slow == 150.0                       # the max over ranks, on every rank
        assert rate == pytest.approx(2 * 81920 / 0.150)
        assert e2e == 2.0


def test_without_a_process_group_the_rank_is_the_job():
    import bench
    assert bench.slowest_rank(12.5) == 12.5
    assert bench.whole_job_rate(81920, 1, 0.2) == pytest.approx(409600.0)


def test_reference_arm_extra_ranks_leave_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
