"""Multi-GPU plumbing: one process per GPU, frames sharded across ranks.

Frames of a batch are independent (every stage is per frame and film-grain
seeds are per frame), so N GPUs filter N disjoint shards with no collective
on the data path; torch.distributed is used only to line the ranks up and to
take the slowest rank's time (weak scaling: every rank keeps the per-rank
batch size).
"""

import datetime
import os


def env():
    """(rank, world size, local rank) from the launcher's environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def init(backend, timeout_s=120):
    """Joins the process group (127.0.0.1 rendezvous from the launcher)."""
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def shard(n_per_rank, rank):
    """This rank's frame indices: a contiguous block, disjoint across ranks."""
    return range(rank * n_per_rank, (rank + 1) * n_per_rank)


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value, world, device="cpu"):
    """The largest value over all ranks (the job's time is its slowest rank's)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
