"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): the HMVM runs as
independent replicas, and the reported time is the slowest rank's."""
import os
import sys

import pytest
import torch.multiprocessing as mp

from helpers import ROOT


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 1.5 + rank  # rank 1 is slower
        q.put((rank, bench.max_over_ranks(mine, dist, torch.device("cpu")),
               bench.max_over_ranks(mine, None, torch.device("cpu"))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.5, 1.5), (1, 2.5, 2.5)]


def test_reference_arm_runs_on_rank0_only(tmp_path):
    import subprocess

    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "2000",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
