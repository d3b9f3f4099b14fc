"""The host side of bench.py's multi-GPU path on CPU: world size 2 over gloo.

The path shards by replica (each rank reconstructs its own volume, no data
exchange); what the ranks share is the timing: every rank takes the maximum
of the per-rank device times with one all-reduce, and rank 0 reports the
whole-job rate. The reference arm and the batch/serving configs run on rank 0
only; the other ranks must exit 0 without work.
"""
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


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r was slower on the first timing and faster on the second
        got = bench.max_over_ranks(dist, [10.0 + rank, 5.0 - rank], "cpu")
        dist.barrier()
        q.put((rank, got, bench.replica_throughput(world, 1000.0, got[0])))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, got, rate in res:
        assert got == [11.0, 5.0]
        assert rate == pytest.approx(2 * 1000.0 / 11e-3)


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, [1, 2.5], "cpu") == [1.0, 2.5]


@pytest.mark.parametrize("args", [["--impl", "reference"], ["--config", "batch"], ["--config", "serving"],
                                  ["--config", "batch", "--impl", "reference"]])
def test_non_zero_rank_exits_without_work(args):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "1", "--warmup", "3", *args],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
