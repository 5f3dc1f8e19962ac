"""Replica runs (one reconstruction per GPU, no collective on the data path):
process-group set-up, barrier and the max-over-ranks timing reduction.
Backend "nccl" on GPUs; "gloo" works on CPU (tests)."""
from __future__ import annotations

import datetime
import os


def init(backend: str | None = None, timeout_s: int = 300):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend or "nccl",
                                    timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def finalize(ws: int):
    """Every rank, after its last collective: barrier, then tear the group down."""
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, ws: int) -> float:
    """Largest value over ranks (the slowest rank's time)."""
    if ws == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v: float, ws: int) -> float:
    if ws == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
