"""GPU tests of trigger post-processing (fip_locate_transients) and of the
command line's additions: the preprocessing tool's combined input file and
the --locations table.

The locate rule has no reference code (the reference names its output
locations.fits, README.md:41, and writes the raw tLISI matrix); the checker is
oracle.locate, a plain restatement of the rule.  Tiles and tLISI values must
be identical; refined positions within 1e-4 pixel and 1e-9 rad.
"""
import subprocess

import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import fits, synthetic
import oracle

pytestmark = pytest.mark.gpu


def check_against_oracle(got, found, t, n, tile, cell, thr):
    want = oracle.locate(t, n, tile, cell, thr)
    assert found == len(want)
    assert len(got) == min(found, len(got))
    for g, w in zip(got, want):
        assert (int(g["tile_row"]), int(g["tile_col"])) == (w[0], w[1])
        assert float(g["tlisi"]) == np.float32(w[2])
        assert abs(float(g["row"]) - w[3]) <= 1e-4 and abs(float(g["col"]) - w[4]) <= 1e-4
        assert abs(float(g["x"]) - w[5]) <= 1e-9 and abs(float(g["y"]) - w[6]) <= 1e-9


def test_planted_minima_ties_and_nan(cuda):
    import torch
    rng = np.random.default_rng(4)
    u, tile, n, cell = 32, 16, 512, 2.9e-5
    t = (1.0 - 1e-4 * rng.random((u, u))).astype(np.float32)
    t[5, 7] = 0.5          # a clear minimum
    t[20, 20] = t[20, 21] = 0.7  # a tie: the lower index wins
    t[0, 31] = 0.8         # at the border
    t[10, 10] = np.nan     # never qualifies, ignored as a neighbour
    t[10, 11] = 0.9
    d = torch.tensor(t.reshape(-1), device=cuda)
    got, found = fip.locate_transients(d, n, tile, cell, threshold=0.95, max_out=16)
    check_against_oracle(got, found, t, n, tile, cell, 0.95)
    tiles = [(int(g["tile_row"]), int(g["tile_col"])) for g in got]
    assert tiles == [(5, 7), (20, 20), (0, 31), (10, 11)]
    # max_out smaller than the number found: the deepest ones, and the count.
    got2, found2 = fip.locate_transients(d, n, tile, cell, threshold=0.95, max_out=2)
    assert found2 == 4 and [(int(g["tile_row"]), int(g["tile_col"])) for g in got2] == tiles[:2]


def test_headline_transient_is_located(cuda):
    """4096^2, 130,816 baselines, tile 32, transient in the third snapshot:
    the deepest location is the transient's tile, and its refined position
    lies within a tile of where the synthetic sky put the source (image rows
    follow l, columns follow -m in this imager's orientation)."""
    import torch
    snap = synthetic.config_reference(transient_snapshot=2)
    n, t, cell = snap.image_size, snap.unit_size, snap.cell_size
    res = fip.FIpipe(snap.vis_re, snap.vis_im, snap.B, snap.V, snap.num_baselines, n, 3, cell, t)
    got, found = fip.locate_transients(torch.tensor(res.reshape(-1), device=cuda), n, t, cell,
                                       threshold=0.99)
    check_against_oracle(got, found, res, n, t, cell, 0.99)
    assert found >= 1
    best = got[0]
    assert (int(best["tile_row"]), int(best["tile_col"])) == np.unravel_index(np.argmin(res),
                                                                              res.shape)
    l, m = snap.transient_lm
    assert abs(float(best["row"]) - (n / 2 + 1 + l / cell)) <= t
    assert abs(float(best["col"]) - (n / 2 + 1 - m / cell)) <= t


def _write_separate(snap, tmp_path):
    p = {k: str(tmp_path / f"{k}.fits") for k in ("vr", "vi", "B", "V")}
    fits.write_image(p["vr"], snap.vis_re[:, None])
    fits.write_image(p["vi"], snap.vis_im[:, None])
    fits.write_image(p["B"], snap.B.reshape(-1, 2))
    fits.write_image(p["V"], snap.V.reshape(-1, 3))
    return p


def test_cli_combined_input_and_locations(cuda, tmp_path):
    """The combined file (zero-padded snapshots, padding counted in nb) gives
    the same tLISI as the separate files, and --locations writes the table
    fip_locate_transients returns."""
    snap = synthetic.config_tiny(flag_fraction_max=0.3, transient_snapshot=2, seed=9)
    nb, n, t, cell = snap.num_baselines, snap.image_size, snap.unit_size, snap.cell_size
    p = _write_separate(snap, tmp_path)
    comb = str(tmp_path / "input.fits")
    fits.write_combined(comb, snap.vis_re, snap.vis_im, snap.B, snap.V, 3)
    out_a, out_b = str(tmp_path / "a.fits"), str(tmp_path / "b.fits")
    loc = str(tmp_path / "locations.fits")
    ra = subprocess.run([fip.CLI_PATH, p["vr"], p["vi"], p["B"], p["V"], str(n), str(nb),
                         str(snap.frequency_hz), repr(cell), "3", str(t), out_a],
                        capture_output=True, text=True, timeout=300)
    assert ra.returncode == 0, ra.stderr
    rb = subprocess.run([fip.CLI_PATH, "--combined", comb, str(n), repr(cell), str(t), out_b,
                         "--locations", loc, "--threshold", "0.999"],
                        capture_output=True, text=True, timeout=300)
    assert rb.returncode == 0, rb.stderr
    a, b = fits.read_image(out_a), fits.read_image(out_b)
    # Two processes: the gridder's fixed-point scale per work item follows the
    # binning's (atomic) entry order, so the sums may differ in the last bits.
    assert np.abs(a - b).max() <= 1e-6
    table = fits.read_table(loc)
    want = oracle.locate(b, n, t, cell, 0.999)
    assert len(table["TLISI"]) == len(want) >= 1
    assert [(int(r), int(c)) for r, c in zip(table["TILE_ROW"], table["TILE_COL"])] == \
        [(w[0], w[1]) for w in want]
    assert np.array_equal(table["TLISI"], np.float32([w[2] for w in want]))
