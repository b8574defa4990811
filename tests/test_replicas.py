"""Multi-rank host logic on CPU (gloo, world size 2, rendezvous on
127.0.0.1): the throughput of independent replicas is the units of all
ranks over the slowest rank's time, agreed by every rank; the reference arm
runs on rank 0 only and the other ranks leave without work."""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from icarat2_b200.replicas import job_rate  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r timed 10 (r + 1) ms for 5 design iterations
        value, ms = job_rate(10.0 * (rank + 1), 5, world, dist, "cpu")
        out[rank] = (value, ms)
    finally:
        dist.destroy_process_group()


def test_job_rate_single_rank():
    value, ms = job_rate(20.0, 4)
    assert ms == 20.0 and value == pytest.approx(200.0)
    with pytest.raises(ValueError):
        job_rate(0.0, 4)


def test_job_rate_is_the_slowest_rank_over_two_gloo_ranks():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        value, ms = res[r]
        assert ms == 20.0  # the slower rank's total, on every rank
        assert value == pytest.approx(world * 5 / 0.020)


def test_reference_arm_leaves_other_ranks_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
