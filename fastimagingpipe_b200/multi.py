"""Multi-GPU plumbing for the imaging + trigger path.

The path has no exchange step between snapshot streams: every beam is
independent through imaging, and its trigger needs only its own last three
images.  Scaling across GPUs is therefore by beam, one process per GPU
(torch.distributed for the plumbing), with no collective on the data path;
the only collectives are the timing/throughput reductions below.
"""
from __future__ import annotations

from typing import List, Sequence


def beams_for_rank(n_beams: int, world: int, rank: int) -> List[int]:
    """Round-robin assignment of beams to ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    return [b for b in range(n_beams) if b % world == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. the timed seconds) over all ranks."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_throughput(units_per_rank: Sequence[float], seconds_per_rank: Sequence[float]) -> float:
    """Units processed by all ranks divided by the slowest rank's time."""
    return float(sum(units_per_rank)) / max(seconds_per_rank)
