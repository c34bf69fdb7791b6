"""The N > 1 path of bench.py on CPU: two gloo ranks in spawned processes.

Multi-GPU runs are replicas (every rank tracks its own seeded pair, no
collective on the data path); the only cross-rank step is the max-over-ranks
time, and only rank 0 prints.  The reference arm does its work on rank 0
alone; the other ranks exit 0 at once.
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(torch, 10.0 + 5.0 * rank, world, "cpu")  # rank 1 is the slow one
        q.put((rank, ms, bench.replica_seed(rank), bench.job_rate(world, 1000, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_seeds_with_two_gloo_ranks():
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
    assert [r[1] for r in res] == [15.0, 15.0]  # both ranks see the slowest rank's time
    assert res[0][2] != res[1][2]  # each replica tracks its own pair
    assert res[0][3] == 2 * 1000 / 15e-3  # whole-job rate: both ranks' units over the slowest time


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import torch

    import bench
    assert bench.max_over_ranks(torch, 7.0, 1, "cpu") == 7.0


def test_reference_arm_on_a_non_zero_rank_exits_at_once():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
    for ln in r.stdout.splitlines():
        json.loads(ln)
