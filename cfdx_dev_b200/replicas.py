"""Replica bookkeeping for runs of one process per GPU.

The pressure solve does not shard across GPUs: N GPUs run N independent
replicas of the solve (each rank its own seeded right-hand sides) and there is
no collective on the data path.  What the ranks share is the host-side
bookkeeping: the launcher's environment, a disjoint block of right-hand-side
seeds per rank, and the job's time per step -- the slowest rank's, reduced
with a MAX over ranks (a device tensor under NCCL, a CPU tensor under gloo).
"""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(rank, local rank, world size) from the torchrun environment; (0, 0, 1) alone."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def seed_offsets(rank: int, per_rank: int) -> list[int]:
    """Seed offsets of this rank's right-hand sides: ranks take disjoint blocks."""
    if rank < 0 or per_rank <= 0:
        raise ValueError("rank must be >= 0 and per_rank > 0")
    return [rank * per_rank + k for k in range(per_rank)]


def max_over_ranks(values, device=None) -> list[float]:
    """Element-wise maximum of `values` over all ranks (identity without a
    process group).  Every rank must call it, in the same order."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]
