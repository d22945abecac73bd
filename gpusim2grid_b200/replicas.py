"""Replicas across GPUs: one process per GPU (torchrun), every rank solving
its own batch of rows with no collective on the data path -- the rows of a
sweep are independent (the reference partitions them the same way: each
row is its own system).  Collectives appear only around measurement: a
barrier before and after the timed region and the maximum of the ranks'
times.

The backend is NCCL on GPUs and gloo on CPU (the tests run two gloo ranks).
"""

from __future__ import annotations

import datetime
import os

__all__ = ["RankInfo", "rank_info", "init", "shard_rows", "max_over_ranks", "sum_over_ranks", "barrier", "finish"]


class RankInfo:
    def __init__(self, rank, world, local):
        self.rank, self.world, self.local = int(rank), int(world), int(local)

    def __repr__(self):
        return f"RankInfo(rank={self.rank}, world={self.world}, local={self.local})"


def rank_info():
    """Rank, world size and local rank from the torchrun environment (1 process
    when absent)."""
    return RankInfo(os.environ.get("RANK", "0"), os.environ.get("WORLD_SIZE", "1"),
                    os.environ.get("LOCAL_RANK", "0"))


def init(backend="nccl", timeout_s=600):
    """Join the process group when there is more than one rank.  Returns the
    RankInfo.  A short timeout makes a rank that waits for a dead peer end
    with an error instead of hanging."""
    import torch.distributed as dist
    info = rank_info()
    if info.world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return info


def shard_rows(n_rows, rank, world):
    """The contiguous slice [begin, end) of n_rows rows that rank `rank` of
    `world` solves when a batch is split instead of replicated (sizes differ
    by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(n_rows), world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def _reduce(value, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device="cpu"):
    """Maximum of a per-rank number (the timed region of a multi-GPU run is
    the slowest rank's)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value, device="cpu"):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM, device)


def barrier(device_sync=True):
    """Synchronise the local device (when one is in use) and every rank."""
    import torch
    import torch.distributed as dist
    if device_sync and torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finish():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
