"""The replicated (N > 1) bench path on the CPU: two gloo ranks on 127.0.0.1.

bench.py runs one replica of the workload per GPU under torchrun and reports the whole job: the
units all ranks processed over the slowest rank's time. These tests run that reduction with two
processes on gloo, and check that the reference arm prints from rank 0 only.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world_size: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        local_ms = [12.5, 20.0][rank]
        slowest = bench.max_over_ranks(local_ms, dist, "cpu")
        rate = bench.whole_job_rate(1000 * 10, world_size, slowest * 1e-3)
        out.put((rank, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_rank_and_the_whole_job():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate in results:
        assert slowest == 20.0
        assert rate == pytest.approx(2 * 1000 * 10 / 0.020)


def test_the_reference_arm_prints_from_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"], cwd=ROOT,
                          env=env, capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0
    assert proc.stdout.strip() == ""


def test_single_rank_reduction_is_the_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_rate(100, 1, 2.0) == 50.0
