"""Whole-job numbers of independent replicas (one system per GPU, no
data-path collective): the path does not shard, so N GPUs run N copies of the
workload and the job's time is the slowest rank's.  Used by bench.py under
torchrun; the collective is only the final max-reduction of the times."""
from __future__ import annotations


def max_over_ranks(seconds: float, device: str = "cpu") -> float:
    """The largest of every rank's `seconds` (the rank's own value without a
    process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(work_per_rank: float, seconds: float, device: str = "cpu") -> tuple[float, float]:
    """(whole-job rate, max seconds): every rank did work_per_rank in its own
    `seconds`; the job did world * work_per_rank in the slowest rank's time."""
    import torch.distributed as dist

    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    t = max_over_ranks(seconds, device)
    return world * work_per_rank / t, t
