"""The multi-rank (replicas) path of bench.py on CPU: two gloo ranks, the
job time is the slowest rank's, the job's throughput counts every rank's
work, and the reference arm runs on rank 0 only.  No GPU."""
import json
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


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        bench.barrier(ws)
        slowest = bench.max_over_ranks(10.0 + rank, ws)  # rank 1 is the slow one
        rate = bench.job_rate(1000.0, 4, slowest, ws)
        q.put((rank, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_and_count_all_work():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, slowest, rate in got:
        assert slowest == 11.0
        # 2 ranks x 1000 units x 4 steps in 11 ms
        assert rate == pytest.approx(2 * 1000 * 4 / 0.011)


def test_reference_arm_prints_nothing_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
