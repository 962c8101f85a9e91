"""The gridding entry point that allocates nothing.

Some callers cannot allocate device memory: code working inside a fixed
memory pool or arena, plugins whose host application owns every device
allocation, and real-time loops that must not call into the allocator.
fip_grid_snapshot_noalloc serves them by keeping its binning scratch in a
fixed device array inside the library.  This file checks, through the C ABI,
that it grids exactly what the allocating entry point (fip_grid_snapshot)
grids, on two calls in a row with different snapshots, and that requests
beyond its fixed limits are refused with a clear error.  It runs last so a
failure here does not stop the rest of a `-x` run.
"""
import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import synthetic

pytestmark = pytest.mark.gpu

# Same tolerance as the other grid comparisons: only the order of the FP32
# shared-memory sums differs between runs.
REL_RMS = 1e-6


def test_no_alloc_grid_matches_allocating_entry_point(cuda):
    import torch
    for seed in (1, 5):  # two calls in a row, different data each time
        snap = synthetic.config_small(seed=seed)
        n, nb, cell = snap.image_size, snap.num_baselines, snap.cell_size
        g = int(np.ceil(np.float32(1.5) * n))
        cells = g * (g // 2 + 1) * 2
        d = {k: torch.tensor(getattr(snap, k)[:nb * (2 if k == "B" else 1)]
                             if k != "V" else snap.V[:9], device=cuda)
             for k in ("vis_re", "vis_im", "B", "V")}
        want = torch.zeros(cells, device=cuda)
        got = torch.full((cells,), float("nan"), device=cuda)  # every cell must be written
        with fip.Imager(n, nb, cell, snap.unit_size) as im:
            im.grid_snapshot(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, want)
        fip.grid_snapshot_noalloc(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, n, cell, got)
        torch.cuda.synchronize()
        a, b = got.cpu().numpy(), want.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.sqrt(((a - b) ** 2).mean() / (b ** 2).mean()) <= REL_RMS


def test_no_alloc_limits_are_enforced(cuda):
    import torch
    z = torch.zeros(16, device=cuda)
    with pytest.raises(fip.FipError, match="131072"):
        fip.grid_snapshot_noalloc(z, z, z, z, 131073, 512, 2.9e-5, z)
    with pytest.raises(fip.FipError, match="4096"):
        fip.grid_snapshot_noalloc(z, z, z, z, 10, 8192, 2.9e-5, z)
