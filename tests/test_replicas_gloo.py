"""The multi-GPU path of bench.py (replicas only: each rank steps its own
channel, no collective on the data path) on CPU: two gloo ranks.

- the timings every rank reports are reduced to their maximum, element by
  element, and every rank sees the same result;
- the whole-job rate counts every rank's points over that maximum;
- the reference arm prints its line on rank 0 only, and the other ranks exit
  0 without work.
"""
import datetime
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r's mixed and FP64 times: the slower rank differs per entry
        mine = [10.0 + rank, 30.0 - 5.0 * rank]
        got = bench.max_over_ranks(mine, torch, dist, device="cpu")
        dist.barrier()
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert res[0] == res[1] == [11.0, 30.0]


def test_max_over_ranks_without_process_group():
    assert bench.max_over_ranks([1.5, 2], torch, None) == [1.5, 2.0]


def test_aggregate_rate_counts_every_replica():
    pts = 256 * 257 * 256
    one = bench.aggregate_rate(pts, 1, 20, 100.0)
    assert one == pytest.approx(pts * 20 / 0.1 / 1e6)
    # weak scaling: N replicas in the same (maximum) time give N times the rate
    assert bench.aggregate_rate(pts, 4, 20, 100.0) == pytest.approx(4 * one)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
