"""Replica timing over ranks (the N > 1 path of bench.py): two gloo ranks on the CPU.

Every rank solves its own replica; the step time is the maximum over ranks and the job's
rate counts both ranks' units.  The reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys
from datetime import timedelta

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hastycompute_b200 import replicas

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        dist.barrier()
        ms = replicas.max_over_ranks(10.0 + rank, dist)  # rank 1 is the slower replica
        q.put((rank, ms, replicas.job_rate(world, 160, ms), replicas.replica_seed(100, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]
    assert out[0][2] == pytest.approx(2 * 160 / 0.011) and out[1][2] == out[0][2]
    assert out[0][3] == 100 and out[1][3] != out[0][3]


def test_one_rank_needs_no_group():
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.job_rate(1, 100, 500.0) == pytest.approx(200.0)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
