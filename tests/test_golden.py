"""Pins the CPU oracle against outputs of the reference's own CUDA build
(tests/golden/*.npz, made by tests/golden/make_golden.py on a B200).

The reference evaluates its pixel mapping through an FP32 fast-math trig
chain and sums with float atomics, so it differs from exact arithmetic; the
tolerances below are the reference's own observed error against the FP64
oracle, with headroom (observed: tiny images 9e-4 relative RMS, maxima 1.3e-3,
targets 0.0027 px, pre-reprojection image 1.2e-6; small tLISI 8.5e-4, maxima
2.0e-3, row/column sums 2.7e-4 relative RMS, crops 3.9e-3, targets 0.0106 px).
"""
import hashlib
import os

import numpy as np
import pytest

import oracle
from fastimagingpipe_b200 import synthetic

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    p = os.path.join(HERE, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated yet (tests/golden/make_golden.py on a GPU)")
    return np.load(p)


def digest(snap):
    h = hashlib.sha256()
    for a in (snap.vis_re, snap.vis_im, snap.B, snap.V):
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    return h.hexdigest()


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).mean() / (b ** 2).mean()))


def test_oracle_pinned_to_reference_tiny():
    g = load("reference_tiny.npz")
    snap = synthetic.config_tiny(transient_snapshot=2)
    assert digest(snap) == str(g["digest"]), "synthetic inputs drifted from the fixture"
    res, imgs, mx = oracle.fipipe(snap, "f64", want_images=True)
    for k in range(3):
        assert relrms(imgs[k], g["images"][k]) < 3e-3
    assert np.allclose(mx, g["maxall"], rtol=5e-3)
    assert np.abs(res - g["tlisi"]).max() < 1e-4
    assert np.array_equal(g["tlisi"], g["tlisi_from_images"])
    tg = oracle.pixel_targets(snap.V[:9], snap.image_size, snap.cell_size, "f64")
    assert np.abs(tg - g["targets0"]).max() < 0.01
    vr, vi, B, V = snap.snapshot(0)
    _, _, pre = oracle.image_snapshot(B, vr, vi, V, snap.num_baselines, snap.image_size,
                                      snap.cell_size, want_pre=True)
    # Before the reprojection the reference differs from exact arithmetic
    # only by FP32 summation, FFT and fast-math taper rounding.
    assert relrms(pre, g["pre0"]) < 2e-5


def test_oracle_pinned_to_reference_small():
    g = load("reference_small.npz")
    snap = synthetic.config_small(transient_snapshot=2)
    assert digest(snap) == str(g["digest"]), "synthetic inputs drifted from the fixture"
    res, imgs, mx = oracle.fipipe(snap, "f64", want_images=True)
    assert np.abs(res - g["tlisi"]).max() < 2e-3
    assert np.unravel_index(np.argmin(res), res.shape) == \
        np.unravel_index(np.argmin(g["tlisi"]), res.shape)
    assert np.allclose(mx, g["maxall"], rtol=5e-3)
    assert relrms(imgs.sum(axis=2), g["row_sums"]) < 1e-3
    assert relrms(imgs.sum(axis=1), g["col_sums"]) < 1e-3
    for k in range(3):
        r0, c0 = g["crop_origins"][k]
        assert relrms(imgs[k][r0:r0 + 64, c0:c0 + 64], g["crops"][k]) < 1e-2
    tg = oracle.pixel_targets(snap.V[:9], snap.image_size, snap.cell_size, "f64")
    pix = g["target_pixels"]
    assert np.abs(tg[pix[:, 0], pix[:, 1]] - g["targets"]).max() < 0.05
