"""Multi-GPU plumbing for the imaging + trigger path.

Beams are independent through imaging, and a beam's trigger needs only its
own last three images.  The bench scales by beam, one process per GPU
(torch.distributed for the plumbing), with no collective on the data path;
the only collectives there are the timing/throughput reductions below.  One
beam's run of snapshots can also be split into contiguous ranges across
ranks (image_range_sharded), whose one exchange step is the two images at
each range boundary.
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


# ---------------------------------------------------------------------------
# Sharding one beam's run of snapshots by contiguous ranges.
#
# The trigger couples three consecutive images, so the only exchange step of
# this sharding is at range boundaries: rank r sends its last two images and
# their maxima to rank r + 1 (point-to-point; NCCL over NVLink on GPUs),
# which then computes the two triples that straddle the boundary in the same
# sliding-window launch as its own.
# ---------------------------------------------------------------------------


def snapshot_range(n_snap: int, world: int, rank: int) -> range:
    """Contiguous range of snapshot indices of `rank` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world or n_snap < 0:
        raise ValueError("invalid rank/world/snapshot count")
    base, extra = divmod(n_snap, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def image_range_sharded(n_snap: int, image_size: int, unit_size: int, image_fn,
                        window_fn, device=None):
    """Images this rank's range of one beam's snapshots and returns the tLISI
    matrices of every triple whose last snapshot lies in the range, as
    {snapshot index: matrix [U, U]}: over all ranks, exactly the sliding-window
    tLISI of the whole run (snapshots 2 .. n_snap - 1).

    image_fn(k, image, image_max) images snapshot k into the flat tensor
    `image` ([N*N]) and `image_max` ([1]); window_fn(images, maxima, count,
    results) writes the sliding-window tLISI of `count` consecutive images
    ([count, N*N], [count]) to results ([count - 2, U*U]) -- on GPUs
    Imager.image_snapshot and Imager.trigger_window.  Ranks exchange only the
    two images at each range boundary (torch.distributed point-to-point);
    every rank needs at least two snapshots.  Without an initialised process
    group the whole run is one range."""
    import torch
    import torch.distributed as dist
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if dist_on else 1
    rank = dist.get_rank() if dist_on else 0
    if n_snap < 2 * world:
        raise ValueError("each rank needs at least two snapshots of the run")
    mine = snapshot_range(n_snap, world, rank)
    n2, u = image_size * image_size, image_size // unit_size
    # Slots 0, 1: the previous range's last two images (received), then ours.
    have_prev = rank > 0
    images = torch.zeros((len(mine) + 2, n2), dtype=torch.float32, device=device)
    maxima = torch.zeros(len(mine) + 2, dtype=torch.float32, device=device)
    for j, k in enumerate(mine):
        image_fn(k, images[j + 2], maxima[j + 2:j + 3])
    if dist_on:
        # Every rank takes the same point-to-point steps in the same order:
        # post the receive from the previous rank, then send to the next.
        reqs = []
        if have_prev:
            reqs.append(dist.irecv(images[0:2], src=rank - 1))
            reqs.append(dist.irecv(maxima[0:2], src=rank - 1))
        if rank + 1 < world:
            reqs.append(dist.isend(images[-2:].contiguous(), dst=rank + 1))
            reqs.append(dist.isend(maxima[-2:].contiguous(), dst=rank + 1))
        for r in reqs:
            r.wait()
    first = 0 if have_prev else 2  # the run's first slot with images
    count = len(mine) + 2 - first
    out = {}
    if count >= 3:
        res = torch.zeros((count - 2, u * u), dtype=torch.float32, device=device)
        window_fn(images[first:], maxima[first:], count, res)
        # Triple i of the window ends in slot first + i + 2, snapshot
        # mine.start + first + i.
        for i in range(count - 2):
            out[mine.start + first + i] = res[i].reshape(u, u)
    return out
