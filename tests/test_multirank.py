"""The replicas path of bench.py --gpus N on CPU: two gloo ranks, each with its
own timed seconds and work, aggregate to the slowest rank's time and the sum
of the work (the whole-job value); the reference arm's non-zero ranks exit
without work.  No GPU."""
import datetime
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path[:0] = [ROOT, os.path.join(ROOT, "autodock-gpu_b200")]
    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        t, w = bench.rank_aggregate(1.5 + rank, 1000.0 * (rank + 1), torch.device("cpu"), world)
        q.put((rank, t, w))
    finally:
        torch.distributed.destroy_process_group()


def test_rank_aggregate_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, w in got:
        assert t == 2.5 and w == 3000.0      # max of the times, sum of the work, on every rank


def test_rank_aggregate_single_process():
    sys.path[:0] = [ROOT, os.path.join(ROOT, "autodock-gpu_b200")]
    import bench
    assert bench.rank_aggregate(2.0, 7.0, None, 1) == (2.0, 7.0)


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
