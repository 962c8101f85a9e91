"""GPU parity at the headline shape: 4096 x 4096 images, 130,816 baselines,
tile 32 (128 x 128 tLISI), and the batching form's mixed-size multi-channel
input (2048^2 and 4096^2, 8 channels over 130-150 MHz, 0-30 % flagged).

Checkers: the reference's own CUDA build (oracle/_ref, run live) and the FP64
CPU oracle (oracle/fip_oracle.c).  Tolerances:
* plain form vs the reference: every image <= 1e-5 relative RMS, maxima
  <= 1e-5 relative, tLISI <= 1e-4 absolute and <= 1e-3 of the matrix's range
  (1 - min tLISI), on a case whose range is large: the transient sits in the
  third snapshot, so D = ||I1-I2| - |I2-I3|| keeps it (1 - tLISI = 0.27 at its
  tile); a transient in the middle snapshot cancels in D and leaves a range of
  1e-4, which no tLISI tolerance can tell from a constant matrix;
* plain form vs FP64: the reference's own error level (images <= 1e-2
  relative RMS, tLISI <= 2e-3), same argmin tile;
* precision form vs FP64: tLISI <= 1e-4 absolute, images <= 3e-5 (FP32
  storage), 2e-4 (FP16), 3e-3 (BF16) relative RMS;
* batching form vs the per-snapshot path: tLISI <= 1e-5 absolute.
"""
import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import synthetic
import oracle
from oracle import reference as ref

from test_gpu_parity import relrms, run

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def third():
    """The headline shape with the transient in the third snapshot."""
    return synthetic.config_reference(transient_snapshot=2)


@pytest.fixture(scope="module")
def third_f64(third):
    return oracle.fipipe(third, "f64", want_images=True)


@pytest.fixture(scope="module")
def flat():
    """The headline shape with every steady source in one quadrant: the other
    three quarters of the sky hold noise alone (near-zero tile variance)."""
    return synthetic.config_reference(transient_snapshot=2, flat_quadrant=True)


def discriminating(want):
    rng = float(1.0 - np.nanmin(want))
    assert rng > 0.1, f"tLISI range {rng}: the case cannot tell a wrong matrix from a right one"
    return rng


def argmin(a):
    return np.unravel_index(np.nanargmin(a), a.shape)


@needs_ref
def test_headline_images_maxima_and_tlisi_match_reference(cuda, third):
    n, nb = third.image_size, third.num_baselines
    res, imgs, mx = run(third, cuda)
    for k in range(3):
        vr, vi, B, V = third.snapshot(k)
        rimg, _, rmx = ref.image_snapshot(vr, vi, B, V, nb, n, third.cell_size)
        assert relrms(imgs[k], rimg) <= 1e-5, f"image {k}"
        assert mx[k] == pytest.approx(rmx, rel=1e-5), f"maximum {k}"
    want = ref.fipipe(third)
    rng = discriminating(want)
    err = float(np.abs(res - want).max())
    assert err <= 1e-4 and err <= 1e-3 * rng
    assert argmin(res) == argmin(want)
    host = fip.FIpipe(third.vis_re, third.vis_im, third.B, third.V, nb, n, 3, third.cell_size,
                      third.unit_size)
    assert np.abs(host - res).max() <= 1e-6


@needs_ref
def test_headline_flat_sky_matches_reference(cuda, flat):
    res, _, _ = run(flat, cuda)
    want = ref.fipipe(flat)
    rng = discriminating(want)
    err = float(np.abs(res - want).max())
    assert err <= 1e-4 and err <= 1e-3 * rng
    assert argmin(res) == argmin(want)


def test_headline_plain_form_vs_fp64(cuda, third, third_f64):
    """The plain form carries the reference's own FP32 error against exact
    arithmetic: its pixel mapping's targets are 0.003-0.05 pixel off, which at
    4096^2 moves the images by 1.7e-2 relative RMS and tLISI by 2.7e-3.
    Bound: no more than the reference build's own error (when it is present)
    plus the plain-vs-reference tolerance; 3e-2 (images) and 5e-3 (tLISI)
    otherwise."""
    res, imgs, mx = run(third, cuda)
    r64, i64, m64 = third_f64
    nb, n = third.num_baselines, third.image_size
    for k in range(3):
        err = relrms(imgs[k], i64[k])
        if ref.available():
            vr, vi, B, V = third.snapshot(k)
            rimg, _, _ = ref.image_snapshot(vr, vi, B, V, nb, n, third.cell_size)
            assert err <= relrms(rimg, i64[k]) * (1 + 1e-3) + 1e-6
        assert err <= 3e-2
    terr = float(np.abs(res - r64).max())
    if ref.available():
        assert terr <= float(np.abs(ref.fipipe(third) - r64).max()) + 1e-4
    assert terr <= 5e-3
    assert argmin(res) == argmin(r64)


@pytest.mark.parametrize("storage,img_tol", [(fip.STORE_F32, 3e-5), (fip.STORE_F16, 2e-4),
                                             (fip.STORE_BF16, 3e-3)])
def test_headline_precision_form_vs_fp64(cuda, third, third_f64, storage, img_tol):
    res, imgs, mx = run(third, cuda, form=fip.FORM_PRECISE, vis_storage=storage)
    r64, i64, m64 = third_f64
    discriminating(r64)
    for k in range(3):
        assert relrms(imgs[k], i64[k]) <= img_tol, f"image {k}"
    assert np.allclose(mx, m64, rtol=img_tol)
    assert np.abs(res - r64).max() <= 1e-4
    assert argmin(res) == argmin(r64)


def test_headline_flat_sky_precision_form_vs_fp64(cuda, flat):
    r64, _, _ = oracle.fipipe(flat, "f64")
    discriminating(r64)
    for storage in (fip.STORE_F16, fip.STORE_BF16):
        res, _, _ = run(flat, cuda, form=fip.FORM_PRECISE, vis_storage=storage)
        assert np.abs(res - r64).max() <= 1e-4
        assert argmin(res) == argmin(r64)


# ---------------------------------------------------------------- batching form

def _fp64_sliding(snaps):
    """FP64 oracle images of MFS snapshots and their sliding-window tLISI."""
    s0 = snaps[0]
    imgs, mx = [], []
    for s in snaps:
        d, m, _ = oracle.image_snapshot(s.B, s.vis_re, s.vis_im, s.V, s.nb, s0.image_size,
                                        s0.cell_size, "f64")
        imgs.append(d)
        mx.append(m)
    return np.stack([oracle.tlisi(imgs[k - 2], imgs[k - 1], imgs[k],
                                  np.array(mx[k - 2:k + 1]), s0.unit_size, "f64")
                     for k in range(2, len(snaps))])


@pytest.mark.parametrize("size", [2048, 4096])
def test_mixed_size_batch_matches_per_snapshot_path_and_fp64(cuda, size):
    """The batching form's configuration: 512 antennas, 8 channels, 0-30 % of
    each snapshot's samples flagged (uneven nb), the cell scaled so both sizes
    see one field of view; 4 snapshots, the transient in the fourth."""
    from test_gpu_batch import batched, dev, per_snapshot
    snaps = synthetic.config_batching(size, n_snap=4, n_chan=8, transient_snapshot=3, seed=2)
    assert len({s.nb for s in snaps}) > 1
    d = dev(snaps, cuda)
    plain_ref = per_snapshot(snaps, d, cuda)
    plain, _ = batched(snaps, d, cuda, [4])
    assert np.abs(plain - plain_ref).max() <= 1e-5
    kw = dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)
    prec, _ = batched(snaps, d, cuda, [4], **kw)
    r64 = _fp64_sliding(snaps)
    assert float(1.0 - r64[-1].min()) > 0.02  # the transient tile stands out
    assert np.abs(prec - r64).max() <= 1e-4
    assert np.abs(plain - r64).max() <= 2e-3
