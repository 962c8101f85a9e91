"""CPU tests of the oracle (oracle/fip_oracle.c) against known answers.

The reference ships no tests or golden vectors; these pin the oracle by
mathematics (independent FFT, quadrature, closed forms, exact tLISI cases)
and, in test_golden.py, by outputs of the reference's own CUDA build.
"""
import math

import numpy as np
import pytest

import oracle
from fastimagingpipe_b200 import synthetic


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 12, 48, 150, 768, 6144])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = oracle.fft1d(x, +1)
    ref = np.fft.ifft(x) * n
    assert np.abs(y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_taper_is_the_es_kernel_transform():
    # taper(t) = 8/norm * integral_0^1 ES(x) cos(8 pi x t / G) dx
    # (FIPkernels.cu:173-186 evaluates it with a 14-node quadrature).
    from scipy.integrate import quad
    n = 512
    g = oracle.grid_size(n)
    tap = oracle.taper(n)
    beta, norm = 15.3704324328, 2.4937047051153827
    es = lambda x: math.exp(beta * (math.sqrt(1 - x * x) - 1))
    for t in (0, 1, 17, 100, 256):
        integral, _ = quad(lambda x: es(x) * math.cos(8 * math.pi * x * t / g), 0, 1, limit=200)
        assert tap[t] == pytest.approx(8 / norm * integral, rel=2e-6, abs=1e-9)


def test_grid_size_matches_reference_rule():
    assert oracle.grid_size(4096) == 6144
    assert oracle.grid_size(512) == 768
    assert oracle.grid_size(100) == 150


def test_single_visibility_grid_footprint():
    # One visibility: separable ES taps over [ceil(p-4), floor(p+4)] with the
    # checkerboard sign (-1)^(r1+r2), centred at (G/2, G/2) (FIPkernels.cu:197-245).
    n = 64
    g = oracle.grid_size(n)
    cell = np.float32(1e-3)
    B = np.array([3.3 / (cell * g), -2.6 / (cell * g)], np.float32)
    V = np.eye(3, dtype=np.float32).ravel()
    grid = oracle.grid(B, [1.0], [0.5], V, 1, n, float(cell))
    scale = np.float64(np.float32(cell)) * g   # the FP64 oracle forms cell * G in double
    p1, p2 = float(B[0]) * scale, float(B[1]) * scale
    nz = np.argwhere(np.abs(grid) > 0)
    rows = nz[:, 0] - g // 2
    cols = nz[:, 1] - g // 2
    assert rows.min() == math.ceil(p1 - 4) and rows.max() == math.floor(p1 + 4)
    assert cols.min() == math.ceil(p2 - 4) and cols.max() == math.floor(p2 + 4)
    beta = 15.3704324328
    es = lambda x: 0.0 if x * x > 1 else math.exp(beta * (math.sqrt(1 - x * x) - 1))
    for (r, c) in [(3, -3), (4, -2), (1, 0), (6, -5)]:
        want = es((r - p1) / 4) * es((c - p2) / 4) * (-1) ** (r + c)
        got = grid[r + g // 2, c + g // 2]
        assert got.real == pytest.approx(want, rel=1e-12)
        assert got.imag == pytest.approx(0.5 * want, rel=1e-12)


def test_point_source_normalisation_and_splat_conservation():
    # A source of flux S at the phase centre: the corrected pre-reprojection
    # peak is sum_v S / |V00 V11 - V01 V10| (gridding kernel and taper cancel,
    # FIPkernels.cu:188-195, 274-287); the bilinear splat then conserves the
    # flux of every source pixel it keeps (weights sum to 1, FIPkernels.cu:394).
    snap = synthetic.config_tiny(n_sources=0, transient_flux=0.0, noise_sigma=0.0)
    n, nb, cell = snap.image_size, snap.num_baselines, snap.cell_size
    _, _, B, V = snap.snapshot(0)
    S = 2.5
    Vm = V.reshape(3, 3).astype(np.float64)
    w = abs(Vm[0, 0] * Vm[1, 1] - Vm[0, 1] * Vm[1, 0])
    img, mx, pre = oracle.image_snapshot(B, np.full(nb, S, np.float32), np.zeros(nb, np.float32),
                                         V, nb, n, cell, want_pre=True)
    assert pre.max() == pytest.approx(nb * S / w, rel=2e-3)
    tg = oracle.pixel_targets(V, n, cell, "f64")
    keep = (np.abs(tg[..., 0]) < n // 2 - 1) & (np.abs(tg[..., 1]) < n // 2 - 1)
    assert img.sum() == pytest.approx(pre[keep].sum() / nb, rel=1e-10)
    assert mx == img.max()


def test_pixel_mapping_chain_equals_closed_form():
    # The degree-based SIN -> slant-SIN chain (FIPkernels.cu:301-376) in FP64
    # equals LL = P1 - xi z/cell, MM = P2 + eta z/cell, z = 1 - sqrt(1 - rho).
    snap = synthetic.config_small()
    n, cell = snap.image_size, snap.cell_size
    V = snap.V[:9].astype(np.float64).reshape(3, 3)
    tg = oracle.pixel_targets(snap.V[:9], n, cell, "f64")
    j, i = np.mgrid[0:n, 0:n]
    a, b = i - n // 2, j - n // 2
    a22 = abs(np.float64(np.float32(V[2, 2])))
    Vf = snap.V[:9].astype(np.float64).reshape(3, 3)
    P1 = (-Vf[0, 0] * a + Vf[1, 0] * b) / a22
    P2 = (-Vf[0, 1] * a + Vf[1, 1] * b) / a22
    rho = cell ** 2 * ((P1 - 1) ** 2 + (P2 - 1) ** 2)
    z = rho / (1 + np.sqrt(1 - rho))
    xi, eta = Vf[2, 0] / Vf[2, 2], Vf[2, 1] / Vf[2, 2]
    cellf = float(np.float32(cell))
    LL = P1 - xi * z / cellf
    MM = P2 + eta * z / cellf
    assert np.abs(tg[..., 0] - LL).max() < 1e-6
    assert np.abs(tg[..., 1] - MM).max() < 1e-6


def test_identical_snapshots_give_unit_tlisi():
    snap = synthetic.config_tiny()
    nb = snap.num_baselines
    for arr in ("vis_re", "vis_im"):
        a = getattr(snap, arr)
        a[nb:2 * nb] = a[:nb]
        a[2 * nb:] = a[:nb]
    snap.B[2 * nb:4 * nb] = snap.B[:2 * nb]
    snap.B[4 * nb:] = snap.B[:2 * nb]
    snap.V[9:18] = snap.V[:9]
    snap.V[18:] = snap.V[:9]
    res, _, _ = oracle.fipipe(snap, "f64")
    assert np.all(res == 1.0)


def test_zero_visibilities_give_nan_like_reference():
    # All-zero visibilities: max over the images is 0 and the combine is
    # 0/0 (FIPkernels.cu:550).
    snap = synthetic.config_tiny()
    snap.vis_re[:] = 0
    snap.vis_im[:] = 0
    res, imgs, mx = oracle.fipipe(snap, "f64", want_images=True)
    assert np.all(mx == 0)
    assert np.all(np.isnan(res))


def test_transient_in_last_snapshot_is_localised():
    snap = synthetic.config_small(transient_snapshot=2)
    res, imgs, _ = oracle.fipipe(snap, "f64", want_images=True)
    d = np.abs(np.abs(imgs[0] - imgs[1]) - np.abs(imgs[1] - imgs[2]))
    peak = np.unravel_index(np.argmax(d), d.shape)
    tile = (peak[0] // snap.unit_size, peak[1] // snap.unit_size)
    assert np.unravel_index(np.argmin(res), res.shape) == tile
    assert 1 - res.min() > 0.1


def test_transient_in_middle_snapshot_cancels():
    # D = ||I1 - I2| - |I2 - I3|| cancels a transient present only in I2.
    snap = synthetic.config_small(transient_snapshot=1)
    res, _, _ = oracle.fipipe(snap, "f64")
    assert 1 - res.min() < 1e-4


def test_f32_restatement_tracks_f64():
    snap = synthetic.config_tiny(transient_snapshot=2)
    r64, i64, m64 = oracle.fipipe(snap, "f64", want_images=True)
    r32, i32, m32 = oracle.fipipe(snap, "f32", want_images=True)
    for k in range(3):
        rel = np.sqrt(((i32[k] - i64[k]) ** 2).mean() / (i64[k] ** 2).mean())
        assert rel < 5e-3
    assert np.abs(r32 - r64).max() < 1e-4


def test_plane_fit_matches_numpy_and_pca():
    snap = synthetic.config_tiny()
    uvw = snap.uvw_m[0]
    B, V = oracle.plane_fit(uvw, [snap.frequency_hz])
    sc = np.float64(np.float32(snap.frequency_hz)) / synthetic.C_LIGHT
    Bn, Vn = synthetic.plane_fit(uvw.astype(np.float64) * sc)
    assert np.allclose(V, Vn, atol=1e-9)
    assert np.allclose(B, Bn, rtol=1e-9, atol=1e-6)
    # SVD_MFS.py:60-110: PCA(2) components, Bin = transform(D) + mean . V
    # equals the uncentred projection (up to each component's sign).
    from sklearn.decomposition import PCA
    D = uvw.astype(np.float64) * sc
    pca = PCA(2).fit(D)
    Bp = pca.transform(D) + D.mean(axis=0) @ pca.components_.T
    for c in range(2):
        s = np.sign(np.dot(pca.components_[c], V[c]))
        assert np.allclose(s * pca.components_[c], V[c], atol=1e-8)
        assert np.allclose(s * Bp[:, c], B[:, c], rtol=1e-8, atol=1e-6)
    assert np.allclose(V @ V.T, np.eye(3), atol=1e-12)


def test_plane_fit_sample_order_and_sign_rule():
    rng = np.random.default_rng(4)
    rows, chans = 50, 3
    uvw = rng.standard_normal((rows, 3)).astype(np.float32) * 100
    uvw[:, 2] *= 0.01
    freqs = np.array([130e6, 140e6, 150e6], np.float32)
    B, V = oracle.plane_fit(uvw, freqs)
    # sample s = row + chan * rows (SVDPreprocessMain.cpp:36-38)
    s = 7 + 2 * rows
    x = uvw[7].astype(np.float64) * (np.float64(freqs[2]) / 299792458.0)
    assert np.allclose(B[s], [x @ V[0], x @ V[1]], rtol=1e-9)
    for c in range(2):
        assert V[c][np.argmax(np.abs(V[c]))] > 0
    assert np.allclose(V[2], np.cross(V[0], V[1]))


def test_collapse_matches_reference_formula():
    rng = np.random.default_rng(5)
    ns = 1000
    v0r, v0i, v3r, v3i = (rng.standard_normal(ns).astype(np.float32) for _ in range(4))
    f0 = rng.random(ns) < 0.2
    f3 = rng.random(ns) < 0.2
    w0 = rng.random(ns).astype(np.float32)
    w3 = rng.random(ns).astype(np.float32)
    w3[:10] = 0
    f0[:10] = True
    o_re, o_im = oracle.collapse(v0r, v0i, v3r, v3i, f0, f3, w0, w3)
    a = np.where(f0, 0.0, w0)
    b = np.where(f3, 0.0, w3)
    ws = a + b
    safe = np.where(ws > 0, ws, 1.0)
    want_re = np.where(ws > 0, (v0r * a + v3r * b) / safe, 0.0)
    want_im = np.where(ws > 0, (v0i * a + v3i * b) / safe, 0.0)
    assert np.allclose(o_re, want_re, atol=1e-6)
    assert np.allclose(o_im, want_im, atol=1e-6)
    assert np.all(o_re[:10] == 0)


def test_locate_rule_known_answers():
    """The locate rule: strict 3 x 3 minima below the threshold, ties to the
    lower index, NaN never a location; centroid refinement in tile units."""
    t = np.ones((8, 8), np.float32)
    t[2, 3] = 0.5
    t[2, 4] = 0.75   # a neighbour of the minimum, not a location itself
    t[6, 6] = t[6, 7] = 0.9
    t[0, 0] = np.nan
    loc = oracle.locate(t, 128, 16, 1e-3, 0.95)
    assert [(r, c) for r, c, *_ in loc] == [(2, 3), (6, 6)]
    r, c, v, row, col, x, y = loc[0]
    # drops 0.5 at (2,3) and 0.25 at (2,4): the column moves a third of a tile
    assert v == np.float32(0.5) and row == 2 * 16 + 7.5
    assert abs(col - ((3 + 0.25 / 0.75) * 16 + 7.5)) < 1e-9
    assert abs(x + 1e-3 * (col - 65)) < 1e-12 and abs(y - 1e-3 * (row - 65)) < 1e-12
