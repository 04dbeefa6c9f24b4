"""Multi-GPU plumbing for the replica runs: one process per GPU, no data-path
collective (every configuration fits one B200).  Only timing is reduced
across ranks (max).  ``shard`` gives the deterministic contiguous partition
of independent items (batched cases) over ranks for a caller that splits
them; the benchmark runs identical replicas and does not split.
"""

from __future__ import annotations

import os


def world() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items: int, rank: int, world_size: int) -> list[int]:
    """Items of `rank` under a contiguous, balanced partition (sizes differ by
    at most one; every item on exactly one rank)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"bad rank {rank} of {world_size}")
    base, extra = divmod(n_items, world_size)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return list(range(start, stop))


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity when not
    distributed).  Every rank must call it at the same point."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]
