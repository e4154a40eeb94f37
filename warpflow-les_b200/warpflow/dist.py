"""Process-per-GPU helpers.

A single cavity case does not shard across GPUs (the reference's domain
decomposition changes the red-black sweep results at sub-domain seams), so
multi-GPU runs are replicas: independent cases are dealt out to ranks and
the only collectives are the timing barrier and a max/sum of scalars.
"""
from __future__ import annotations

import os

import torch


def world():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank, size):
    """Deal items round-robin: rank r gets items r, r+size, ..."""
    return list(items)[rank::size]


def _reduce(value, op, device):
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device="cpu"):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value, device="cpu"):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM, device)
