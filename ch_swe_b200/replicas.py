"""Replica runs on several GPUs of one node (one process per GPU, launched by
torchrun): every rank integrates its own members, no collective touches the
data path; only the timing is combined (max over ranks) and results may be
gathered on the host.  The backend is NCCL on GPUs and gloo in CPU tests."""
from __future__ import annotations

import os
from datetime import timedelta


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, local_rank: int = 0, timeout_s: float = 120.0):
    import torch
    import torch.distributed as dist
    kw = {"timeout": timedelta(seconds=timeout_s)}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(value: float, dist, device: str = "cpu") -> float:
    """Maximum of a per-rank float (the slowest rank's time)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist, device: str = "cpu") -> float:
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
