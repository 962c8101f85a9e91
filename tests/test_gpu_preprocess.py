"""GPU tests of on-device preprocessing ahead of the imager.

* The flag/weight Stokes-I collapse fused into the gridder's visibility load
  (fip_image_snapshot_raw) against the two-step path (fip_collapse_visibilities,
  then fip_image_snapshot): images within 1e-6 relative RMS (only the order
  of the gridder's fixed-point sums may differ), maxima within 1e-6.
* The whole chain from raw data -- uvw in metres and channel frequencies
  through the device plane fit (fip_plane_project, sample order row + chan *
  rows) and the fused collapse into the image -- against the FP64 oracle's
  plane fit, collapse and imager: images within 1e-4 relative RMS (precision
  form; the device fit's FP32 outputs against the FP64 fit).
* The device plane fit and collapse against the reference's own GPU
  preprocessing (SVDPreprocessKernels.cu recompiled for sm_100a,
  oracle/_ref/libfippre.so: FP32 moments with atomics, a cuSOLVER
  eigensolve, its PCA sign rule), run live: V and B within the FP32
  covariance's rounding, the collapsed visibilities within 1e-6.
"""
import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import synthetic
import oracle
from oracle import reference as ref

pytestmark = pytest.mark.gpu
needs_pre = pytest.mark.skipif(not ref.preprocess_available(),
                               reason="oracle/_ref/libfippre.so not built")


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).mean() / (b ** 2).mean()))


def raw_device(raw, cuda):
    import torch
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=cuda)
    return dict(v0_re=t(raw.xx.real.astype(np.float32)), v0_im=t(raw.xx.imag.astype(np.float32)),
                v3_re=t(raw.yy.real.astype(np.float32)), v3_im=t(raw.yy.imag.astype(np.float32)),
                flag0=t(raw.flag0), flag3=t(raw.flag3), weight0=t(raw.weight0),
                weight3=t(raw.weight3))


def plane(raw, cuda):
    import torch
    rows, chans = raw.uvw_m.shape[0], raw.freqs_hz.shape[0]
    B = torch.zeros(rows * chans * 2, device=cuda)
    V = torch.zeros(9, device=cuda)
    fip.plane_project(torch.tensor(raw.uvw_m.reshape(-1), device=cuda),
                      torch.tensor(raw.freqs_hz, device=cuda), rows, chans, B, V)
    return B, V


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE),
                                dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)])
def test_fused_collapse_matches_collapse_then_image(cuda, kw):
    import torch
    raw = synthetic.make_raw_snapshot()
    n, ns = raw.image_size, raw.num_samples
    d = raw_device(raw, cuda)
    B, V = plane(raw, cuda)
    cre, cim = torch.zeros(ns, device=cuda), torch.zeros(ns, device=cuda)
    fip.collapse_visibilities(d["v0_re"], d["v0_im"], d["v3_re"], d["v3_im"], d["flag0"],
                              d["flag3"], d["weight0"], d["weight3"], cre, cim, ns)
    two = torch.zeros(n * n, device=cuda)
    fused = torch.full((n * n,), float("nan"), device=cuda)
    m2, mf = torch.zeros(1, device=cuda), torch.zeros(1, device=cuda)
    with fip.Imager(n, ns, raw.cell_size, 16, **kw) as im:
        im.image_snapshot(cre, cim, B, V, ns, two, m2)
        im.image_snapshot_raw(d["v0_re"], d["v0_im"], d["v3_re"], d["v3_im"], d["flag0"],
                              d["flag3"], d["weight0"], d["weight3"], B, V, ns, fused, mf)
        torch.cuda.synchronize()
        im.check()
    a, b = fused.cpu().numpy(), two.cpu().numpy()
    assert np.isfinite(a).all()
    assert relrms(a, b) <= 1e-6
    assert float(mf.item()) == pytest.approx(float(m2.item()), rel=1e-6)


def test_raw_data_to_image_on_device_vs_fp64_oracle(cuda):
    import torch
    raw = synthetic.make_raw_snapshot(seed=11)
    n, ns = raw.image_size, raw.num_samples
    d = raw_device(raw, cuda)
    B, V = plane(raw, cuda)
    img = torch.zeros(n * n, device=cuda)
    with fip.Imager(n, ns, raw.cell_size, 16, form=fip.FORM_PRECISE) as im:
        im.image_snapshot_raw(d["v0_re"], d["v0_im"], d["v3_re"], d["v3_im"], d["flag0"],
                              d["flag3"], d["weight0"], d["weight3"], B, V, ns, img)
        torch.cuda.synchronize()
    # Oracle: FP64 plane fit, FP64 collapse, FP64 imager.
    Bo, Vo = oracle.plane_fit(raw.uvw_m, raw.freqs_hz)
    cre, cim = oracle.collapse(raw.xx.real, raw.xx.imag, raw.yy.real, raw.yy.imag, raw.flag0,
                               raw.flag3, raw.weight0, raw.weight3)
    want, _, _ = oracle.image_snapshot(Bo.reshape(-1).astype(np.float32), cre, cim,
                                       Vo.reshape(-1).astype(np.float32), ns, n, raw.cell_size,
                                       "f64")
    assert relrms(img.cpu().numpy().reshape(n, n), want) <= 1e-4


def test_raw_entry_point_rejects_null_arrays(cuda):
    import torch
    z = torch.zeros(64, device=cuda)
    u8 = torch.zeros(64, dtype=torch.uint8, device=cuda)
    with fip.Imager(64, 64, 1e-3, 16) as im:
        with pytest.raises(fip.FipError):
            im.image_snapshot_raw(z, z, z, z, u8, None, z, z, z, z, 64, z)


@needs_pre
@pytest.mark.parametrize("seed,ha,chans", [(7, 1.5, (130e6, 140e6, 150e6)),
                                           (12, -2.0, (142e6,)),
                                           (5, 0.3, tuple(130e6 + 2.5e6 * k for k in range(8)))])
def test_plane_fit_and_collapse_vs_reference_gpu_preprocessing(cuda, seed, ha, chans):
    import torch
    raw = synthetic.make_raw_snapshot(seed=seed, hour_angle_h=ha, freqs_hz=chans)
    ns = raw.num_samples
    B, V = plane(raw, cuda)
    d = raw_device(raw, cuda)
    cre, cim = torch.zeros(ns, device=cuda), torch.zeros(ns, device=cuda)
    fip.collapse_visibilities(d["v0_re"], d["v0_im"], d["v3_re"], d["v3_im"], d["flag0"],
                              d["flag3"], d["weight0"], d["weight3"], cre, cim, ns)
    torch.cuda.synchronize()
    Br, Vr, vr, vi = ref.preprocess(raw.uvw_m, raw.freqs_hz, raw.xx, raw.yy, raw.flag0,
                                    raw.flag3, raw.weight0, raw.weight3)
    got_V = V.cpu().numpy().reshape(3, 3)
    # Same rows, signs and handedness (the sign rule picks each row's sign
    # from its largest component; the third row is their cross product).
    assert np.abs(got_V - Vr).max() <= 2e-5, (got_V, Vr)
    got_B = B.cpu().numpy().reshape(-1, 2)
    scale = float(np.abs(Br).max())
    assert np.abs(got_B - Br).max() <= 3e-5 * scale
    assert np.allclose(cre.cpu().numpy(), vr, rtol=1e-6, atol=1e-6)
    assert np.allclose(cim.cpu().numpy(), vi, rtol=1e-6, atol=1e-6)
    # The oracle's FP64 fit (the checker of the tests above) against the
    # reference's, pinning its sign rule and sample order.
    Bo, Vo = oracle.plane_fit(raw.uvw_m, raw.freqs_hz)
    assert np.abs(Vo - Vr).max() <= 2e-5
    assert np.abs(Bo - Br).max() <= 3e-5 * scale
