"""One process per GPU, replicas only.

Snapshots are independent, so N GPUs run N independent snapshot streams: each
rank takes its own share of the snapshots and no collective touches the data
path.  The only collectives are a barrier around the timed region and the
max-over-ranks reduction of the elapsed device time.
"""
from __future__ import annotations

import datetime
import os


def env_rank() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 120):
    """Initialise the process group from torchrun's environment (no-op for 1 rank)."""
    rank, world, _ = env_rank()
    if world <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous share of n_items for this rank (sizes differ by at most one)."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar (the job time is the slowest rank's)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist=None):
    if dist is not None:
        dist.barrier()


def finalize(dist=None):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
