"""Multi-process replica path on CPU (gloo, world size 2): the timing reduction the
benchmark uses across GPUs, and the reference arm's rank handling."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from ch_swe_b200 import replicas
    dist = replicas.init("gloo", rank, timeout_s=30)
    mx = replicas.max_over_ranks(10.0 + rank, dist)
    sm = replicas.sum_over_ranks(1.0, dist)
    out[rank] = (mx, sm)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == (11.0, 2.0) and out[1] == (11.0, 2.0)


def test_reference_arm_rank1_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
