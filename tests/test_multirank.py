"""The multi-GPU path of bench.py on CPU: two ranks under a gloo process
group (torch.distributed.run's environment, rendezvous on 127.0.0.1).

Every rank renders its own frame (replicas: the path has no exchange
step), so the only collective is the max over ranks of the timed region;
the whole-job throughput counts every rank's paths over the slowest
rank's time.  The reference arm runs on rank 0 alone.
"""
import datetime
import os
import socket
import subprocess
import sys

import multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, REPO)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        env = bench.rank_env()
        slowest = bench.max_over_ranks(100.0 * (rank + 1), dist, "cpu")
        value = bench.job_throughput(1_000_000, 5, world, slowest)
        q.put((rank, env, slowest, value))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_the_slowest_and_count_every_frame():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, env, slowest, value in got:
        assert env == (2, rank, rank)
        assert slowest == 200.0  # rank 1's 200 ms
        # 2 ranks x 1 M paths x 5 steps in 0.2 s
        assert abs(value - 50.0) < 1e-9


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(123.0, None, "cpu") == 123.0
    assert bench.job_throughput(2_000_000, 4, 1, 1000.0) == 8.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
