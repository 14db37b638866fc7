"""Multi-GPU plumbing for the benchmark: one process per GPU, blocks shard
over ranks with no collective on the data path (each rank correlates its
own blocks), and timings reduce as the max over ranks.  torch.distributed
is used only for the barrier and that reduction (NCCL on GPUs, gloo in the
CPU tests)."""
from __future__ import annotations

import datetime
import os


def world():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items: int, rank: int, world_size: int) -> range:
    """Contiguous, balanced share of n_items for `rank`."""
    lo = n_items * rank // world_size
    hi = n_items * (rank + 1) // world_size
    return range(lo, hi)


def init(backend: str, timeout_s: int = 120):
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank timing over all ranks (identity without a group)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
