"""GPU parity tests of the CUDA path (through the C ABI) against the oracles.

Checkers:
* the reference's own CUDA build (oracle/_ref/libfipref.so), run live when
  present, and its golden fixtures (tests/golden/*.npz);
* the FP64 CPU oracle (oracle/fip_oracle.c).

Tolerances (the project's parity bar):
* plain FP32 form vs the reference: pixel targets bit-identical, images
  <= 1e-5 relative RMS (float-atomic summation order differs), tLISI <= 1e-4
  absolute;
* plain form vs FP64: the reference's own error level (images <= 1e-2
  relative RMS, tLISI <= 2e-3);
* precision form vs FP64: tLISI <= 1e-4 absolute, images <= 1e-4 relative RMS
  (FP32 storage <= 3e-5).
"""
import os
import subprocess

import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import fits, synthetic
import oracle
from oracle import reference as ref

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).mean() / (b ** 2).mean()))


def to_dev(snap, dev):
    import torch
    return {k: torch.tensor(np.ascontiguousarray(getattr(snap, k)), device=dev)
            for k in ("vis_re", "vis_im", "B", "V")}


def run(snap, dev, check=True, **kw):
    """Images the three snapshots and computes the trigger through the C ABI.
    -> (tlisi [U,U], images [3,N,N], maxima [3]).  check: fail if a gather
    tile lay outside the gather's domain."""
    import torch
    n, nb, t = snap.image_size, snap.num_baselines, snap.unit_size
    u = n // t
    d = to_dev(snap, dev)
    imgs = torch.zeros((3, n * n), device=dev)
    mx = torch.zeros(3, device=dev)
    res = torch.zeros(u * u, device=dev)
    with fip.Imager(n, nb, snap.cell_size, t, **kw) as im:
        for k in range(3):
            im.image_snapshot(d["vis_re"][k * nb:], d["vis_im"][k * nb:], d["B"][2 * k * nb:],
                              d["V"][9 * k:], nb, imgs[k], mx[k:])
        im.trigger(imgs[0], imgs[1], imgs[2], mx, res)
        torch.cuda.synchronize()
        if check:
            im.check()  # no gather tile outside its domain
    return (res.cpu().numpy().reshape(u, u), imgs.cpu().numpy().reshape(3, n, n),
            mx.cpu().numpy())


def targets(snap, dev, exact=False, k=0):
    import torch
    n = snap.image_size
    out = torch.zeros(n * n * 2, device=dev)
    V = torch.tensor(snap.V[9 * k:9 * k + 9], device=dev)
    with fip.Imager(n, snap.num_baselines, snap.cell_size, snap.unit_size) as im:
        im.pixel_targets(V, out, exact=exact)
        torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, n, 2)


needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def small():
    return synthetic.config_small(transient_snapshot=2)


@pytest.fixture(scope="module")
def tiny():
    return synthetic.config_tiny(transient_snapshot=2)


# ---------------------------------------------------------------- reference

def test_targets_bit_identical_to_reference_fixture(cuda, tiny):
    g = np.load(os.path.join(GOLDEN, "reference_tiny.npz"))
    assert np.array_equal(targets(tiny, cuda), g["targets0"])


def test_small_against_reference_fixture(cuda, small):
    g = np.load(os.path.join(GOLDEN, "reference_small.npz"))
    res, imgs, mx = run(small, cuda)
    pix = g["target_pixels"]
    tg = targets(small, cuda)
    assert np.array_equal(tg[pix[:, 0], pix[:, 1]], g["targets"])
    assert np.abs(res - g["tlisi"]).max() <= 1e-4
    assert np.allclose(mx, g["maxall"], rtol=1e-5)
    for k in range(3):
        r0, c0 = g["crop_origins"][k]
        assert relrms(imgs[k][r0:r0 + 64, c0:c0 + 64], g["crops"][k]) <= 1e-5
    assert relrms(imgs.sum(axis=2), g["row_sums"]) <= 1e-5
    assert relrms(imgs.sum(axis=1), g["col_sums"]) <= 1e-5


def test_tiny_images_against_reference_fixture(cuda, tiny):
    g = np.load(os.path.join(GOLDEN, "reference_tiny.npz"))
    res, imgs, mx = run(tiny, cuda)
    for k in range(3):
        assert relrms(imgs[k], g["images"][k]) <= 1e-5
    assert np.abs(res - g["tlisi"]).max() <= 1e-4


@needs_ref
@pytest.mark.parametrize("cfg", ["tiny", "small", "fallback96"])
def test_live_reference_parity(cuda, cfg):
    snap = {"tiny": lambda: synthetic.config_tiny(transient_snapshot=2),
            "small": lambda: synthetic.config_small(transient_snapshot=2),
            "fallback96": lambda: synthetic.config_tiny(image_size=96, cell_size=1.6e-4,
                                                        transient_snapshot=2)}[cfg]()
    n, nb = snap.image_size, snap.num_baselines
    assert np.array_equal(targets(snap, cuda, k=1), ref.pixel_targets(snap.V[9:18], n,
                                                                       snap.cell_size))
    res, imgs, mx = run(snap, cuda)
    for k in range(3):
        vr, vi, B, V = snap.snapshot(k)
        rimg, _, rmx = ref.image_snapshot(vr, vi, B, V, nb, n, snap.cell_size)
        assert relrms(imgs[k], rimg) <= 1e-5
        assert mx[k] == pytest.approx(rmx, rel=1e-5)
    assert np.abs(res - ref.fipipe(snap)).max() <= 1e-4


@needs_ref
def test_reference_shape_tlisi_matches_reference(cuda):
    snap = synthetic.config_reference(transient_snapshot=2)
    got = fip.FIpipe(snap.vis_re, snap.vis_im, snap.B, snap.V, snap.num_baselines,
                     snap.image_size, 3, snap.cell_size, snap.unit_size)
    want = ref.fipipe(snap)
    assert np.abs(got - want).max() <= 1e-4
    assert np.unravel_index(np.argmin(got), got.shape) == np.unravel_index(np.argmin(want),
                                                                          got.shape)


# ---------------------------------------------------------------- FP64 oracle

def test_plain_form_vs_fp64(cuda, small):
    res, imgs, mx = run(small, cuda)
    r64, i64, m64 = oracle.fipipe(small, "f64", want_images=True)
    for k in range(3):
        assert relrms(imgs[k], i64[k]) <= 1e-2
    assert np.abs(res - r64).max() <= 2e-3
    assert np.unravel_index(np.argmin(res), res.shape) == np.unravel_index(np.argmin(r64),
                                                                          res.shape)


@pytest.mark.parametrize("storage,img_tol", [(fip.STORE_F32, 3e-5), (fip.STORE_F16, 2e-4),
                                             (fip.STORE_BF16, 3e-3)])
def test_precision_form_vs_fp64(cuda, small, storage, img_tol):
    res, imgs, mx = run(small, cuda, form=fip.FORM_PRECISE, vis_storage=storage)
    r64, i64, m64 = oracle.fipipe(small, "f64", want_images=True)
    for k in range(3):
        assert relrms(imgs[k], i64[k]) <= img_tol
    assert np.abs(res - r64).max() <= 1e-4


@pytest.mark.parametrize("cfg", ["reference", "wide"])
def test_theta_table_targets_identical_to_evaluated_chain(cuda, cfg):
    """The plain form maps pixels through a table of the chain's theta terms;
    every target must carry the same bits as the chain evaluated step by step.
    "reference": the 4096^2 shape (every theta inside the table); "wide": a
    29-degree field, whose outer pixels fall below the table's 80 degrees and
    evaluate."""
    import torch
    snap = (synthetic.config_reference() if cfg == "reference" else
            synthetic.config_tiny(image_size=512, cell_size=1e-3))
    n = snap.image_size
    a = torch.empty(n * n * 2, device=cuda)
    b = torch.empty_like(a)
    with fip.Imager(n, snap.num_baselines, snap.cell_size, snap.unit_size) as im:
        for k in range(3):
            V = torch.tensor(snap.V[9 * k:9 * k + 9], device=cuda)
            im.pixel_targets(V, a)
            im.pixel_targets(V, b, evaluated=True)
            torch.cuda.synchronize()
            assert torch.equal(a.view(torch.int32), b.view(torch.int32))


@pytest.mark.parametrize("ha,radius", [(1.5, 400.0), (4.0, 400.0), (1.5, 1000.0)])
def test_wide_field_gather_matches_scatter_and_reference(cuda, ha, radius):
    """29-degree fields (512^2, cell 1e-3 rad).  At hour angle 4 h the plane is
    tilted by ~50 degrees (xi = 1.27): the slant term bows every tile's
    preimage by most of a pixel and the map contracts by up to 2, so the
    gather's candidate bounds (curvature margin, row chunks, per-tile
    fixed-point scale) are exercised at image level, against the reference's
    own scatter (the source-major path and the reference build) and, for the
    precision form, against FP64.  With a 1 km array the uv coverage runs
    past the grid's edge, whose taps the reference clamps (FIPkernels.cu:
    211-219) and whose first column is the half-plane grid's Nyquist column."""
    snap = synthetic.config_tiny(image_size=512, cell_size=1e-3, hour_angle0_h=ha,
                                 radius_m=radius, transient_snapshot=2)
    n, nb = snap.image_size, snap.num_baselines
    res_g, img_g, mx_g = run(snap, cuda)
    res_s, img_s, mx_s = run(snap, cuda, reproject=fip.REPROJECT_SCATTER)
    for k in range(3):
        assert relrms(img_g[k], img_s[k]) <= 1e-6
    assert np.allclose(mx_g, mx_s, rtol=1e-6)
    assert np.abs(res_g - res_s).max() <= 1e-5
    if ref.available():
        for k in range(3):
            vr, vi, B, V = snap.snapshot(k)
            rimg, _, _ = ref.image_snapshot(vr, vi, B, V, nb, n, snap.cell_size)
            assert relrms(img_g[k], rimg) <= 1e-5
        assert np.abs(res_g - ref.fipipe(snap)).max() <= 1e-4
    res_p, img_p, _ = run(snap, cuda, form=fip.FORM_PRECISE)
    r64, i64, _ = oracle.fipipe(snap, "f64", want_images=True)
    for k in range(3):
        assert relrms(img_p[k], i64[k]) <= 3e-5
    assert np.abs(res_p - r64).max() <= 1e-4


def test_geometry_outside_the_gather_domain(cuda):
    """A 37-degree field with the plane tilted by ~65 degrees: corners of the
    source image lie beyond the horizon of the slant projection, where the
    map is not invertible tile by tile.  The gather flags it (no silent
    image), and FIpipe, whose bases are host arrays, reprojects such snapshots
    with the reference's scatter."""
    snap = synthetic.config_tiny(image_size=256, cell_size=2.5e-3, hour_angle0_h=5.0,
                                 transient_snapshot=2)
    with pytest.raises(fip.FipError, match="domain"):
        run(snap, cuda)
    want, _, _ = run(snap, cuda, reproject=fip.REPROJECT_SCATTER)
    got = fip.FIpipe(snap.vis_re, snap.vis_im, snap.B, snap.V, snap.num_baselines,
                     snap.image_size, 3, snap.cell_size, snap.unit_size)
    assert np.allclose(got, want, atol=1e-6, equal_nan=True)
    if ref.available():
        r = ref.fipipe(snap)
        both = np.isfinite(got) & np.isfinite(r)
        assert np.array_equal(np.isnan(got), np.isnan(r))
        err = float(np.abs(got - r)[both].max())
        assert err <= 1e-4, f"max |tLISI - reference| = {err} at {np.argmax(np.abs(got - r) * both)}"


def test_exact_targets_vs_oracle(cuda, small):
    tg = targets(small, cuda, exact=True)
    o = oracle.pixel_targets(small.V[:9], small.image_size, small.cell_size, "f64")
    assert np.abs(tg - o).max() <= 1e-4


def test_cufft_fallback_size_vs_fp64(cuda):
    snap = synthetic.config_tiny(image_size=100, cell_size=1.5e-4, unit_size=20,
                                 transient_snapshot=2)
    res, imgs, _ = run(snap, cuda, form=fip.FORM_PRECISE)
    r64, i64, _ = oracle.fipipe(snap, "f64", want_images=True)
    for k in range(3):
        assert relrms(imgs[k], i64[k]) <= 3e-5
    assert np.abs(res - r64).max() <= 1e-4


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE)])
@pytest.mark.parametrize("n,cell,t", [(100, 1.5e-4, 20), (1000, 1.5e-5, 20)])
def test_cufft_fallback_lanes_match_single_snapshot_calls(cuda, n, cell, t, kw):
    """Image sides whose grid is not 3 * 2^k transform with cuFFT; each of the
    three concurrent lanes has its own plan, so the three snapshots of a
    pipe_device / pipe_host call must still give the one-at-a-time results."""
    import torch
    snap = synthetic.config_tiny(image_size=n, cell_size=cell, unit_size=t, transient_snapshot=2)
    nb, u = snap.num_baselines, n // t
    ref, _, _ = run(snap, cuda, **kw)
    d = to_dev(snap, cuda)
    got = torch.zeros(u * u, device=cuda)
    with fip.Imager(n, nb, cell, t, **kw) as im:
        for _ in range(2):
            im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, got)
        host = im.pipe_host(snap.vis_re, snap.vis_im, snap.B, snap.V, nb)
        torch.cuda.synchronize()
    assert np.abs(got.cpu().numpy().reshape(u, u) - ref).max() <= 1e-5
    assert np.abs(host - ref).max() <= 1e-5
    if n == 1000 and kw:  # the precision form's bar against the FP64 oracle
        r64, _, _ = oracle.fipipe(snap, "f64")
        assert np.abs(ref - r64).max() <= 1e-4


def hermitian_half_grid(snap, k=0):
    """The oracle's checkerboarded grid (FIPkernels.cu:197-245) as the
    half-plane Hermitian grid fip_grid_snapshot returns."""
    vr, vi, B, V = snap.snapshot(k)
    n = snap.image_size
    g = oracle.grid_size(n)
    gref = oracle.grid(B, vr, vi, V, snap.num_baselines, n, snap.cell_size)
    r = np.arange(g) - g // 2
    checker = np.where((r[:, None] + r[None, :]) % 2 == 0, 1.0, -1.0)
    gw = np.fft.ifftshift(gref * checker)          # gw[r1 mod G, r2 mod G] = g(r1, r2)
    gneg = np.roll(np.flip(gw, (0, 1)), 1, axis=(0, 1))  # g(-r1, -r2)
    h = 0.5 * (gw + np.conj(gneg))
    return h[:, : g // 2 + 1]


@pytest.mark.parametrize("n", [512, 100, "edge"])
def test_grid_stage_vs_oracle(cuda, n):
    """"edge": uv coverage past the grid's edge (128^2, cell 1e-3): taps at
    r2 = -G/2 land on the Nyquist column of both half-plane copies."""
    import torch
    if n == "edge":
        n = 128
        snap = synthetic.config_tiny(image_size=128, cell_size=1e-3)
    else:
        snap = synthetic.config_small() if n == 512 else \
            synthetic.config_tiny(image_size=100, cell_size=1.5e-4, unit_size=20)
    g = oracle.grid_size(n)
    d = to_dev(snap, cuda)
    out = torch.zeros(g * (g // 2 + 1) * 2, device=cuda)
    with fip.Imager(n, snap.num_baselines, snap.cell_size, snap.unit_size) as im:
        im.grid_snapshot(d["vis_re"], d["vis_im"], d["B"], d["V"], snap.num_baselines, out)
        torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.complex64).reshape(g, g // 2 + 1)
    want = hermitian_half_grid(snap)
    err = np.sqrt((np.abs(got - want) ** 2).mean() / (np.abs(want) ** 2).mean())
    assert err <= 1e-5


# ---------------------------------------------------------------- internal consistency

def test_gather_equals_scatter(cuda, small):
    _, a, ma = run(small, cuda)
    _, b, mb = run(small, cuda, reproject=fip.REPROJECT_SCATTER)
    for k in range(3):
        assert relrms(a[k], b[k]) <= 1e-6
    assert np.allclose(ma, mb, rtol=1e-6)


def test_host_and_device_entry_points_agree(cuda, tiny):
    import torch
    res, _, _ = run(tiny, cuda)
    host = fip.FIpipe(tiny.vis_re, tiny.vis_im, tiny.B, tiny.V, tiny.num_baselines,
                      tiny.image_size, 3, tiny.cell_size, tiny.unit_size)
    assert np.abs(host - res).max() <= 1e-6
    d = to_dev(tiny, cuda)
    u = tiny.image_size // tiny.unit_size
    out = torch.zeros(u * u, device=cuda)
    with fip.Imager(tiny.image_size, tiny.num_baselines, tiny.cell_size, tiny.unit_size) as im:
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], tiny.num_baselines, out)
        assert np.abs(im.pipe_host(tiny.vis_re, tiny.vis_im, tiny.B, tiny.V,
                                   tiny.num_baselines) - res).max() <= 1e-6
    assert np.abs(out.cpu().numpy().reshape(u, u) - res).max() <= 1e-6


class _DeviceFloats:
    """A view of n device floats at an address (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3}


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE)])
@pytest.mark.parametrize("cfg", ["small", "reference"])
def test_fused_trigger_bit_identical_to_separate_trigger(cuda, cfg, kw):
    """pipe_device (plain form) computes the trigger's tile statistics inside
    the last reprojection of every 64 x 64 region, in k_trigger's reduction
    order: its tLISI must equal the separate trigger's on the same images bit
    for bit (the precision form keeps the separate pass: the same check)."""
    import torch
    snap = (synthetic.config_small(transient_snapshot=2) if cfg == "small" else
            synthetic.config_reference(transient_snapshot=2))
    n, nb, t = snap.image_size, snap.num_baselines, snap.unit_size
    u = n // t
    d = to_dev(snap, cuda)
    fused = torch.zeros(u * u, device=cuda)
    sep = torch.zeros(u * u, device=cuda)
    with fip.Imager(n, nb, snap.cell_size, t, **kw) as im:
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, fused)
        torch.cuda.synchronize()
        ptrs = [im.image_ptr(k) for k in range(3)]
        imgs = [torch.as_tensor(_DeviceFloats(p, n * n), device=cuda) for p in ptrs]
        mx = torch.stack([torch.clamp(x.max(), min=0.0) for x in imgs])
        im.trigger(ptrs[0], ptrs[1], ptrs[2], mx, sep)
        torch.cuda.synchronize()
    a, b = fused.cpu().numpy(), sep.cpu().numpy()
    assert np.array_equal(a.view(np.int32), b.view(np.int32))
    assert float(1.0 - a.min()) > 0.1  # the transient's tile is in the matrix


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)])
def test_concurrent_lanes_match_single_snapshot_calls(cuda, small, kw):
    """pipe_device / pipe_host image the three snapshots on concurrent lanes;
    back-to-back calls with different inputs must each give the result of the
    one-snapshot-at-a-time path."""
    import torch
    other = synthetic.config_small(transient_snapshot=1, seed=7)
    n, nb, t = small.image_size, small.num_baselines, small.unit_size
    u = n // t
    ref_a, _, _ = run(small, cuda, **kw)
    ref_b, _, _ = run(other, cuda, **kw)
    da, db = to_dev(small, cuda), to_dev(other, cuda)
    ra, rb = torch.zeros(u * u, device=cuda), torch.zeros(u * u, device=cuda)
    with fip.Imager(n, nb, small.cell_size, t, **kw) as im:
        for _ in range(2):
            im.pipe_device(da["vis_re"], da["vis_im"], da["B"], da["V"], nb, ra)
            im.pipe_device(db["vis_re"], db["vis_im"], db["B"], db["V"], nb, rb)
        hb = im.pipe_host(other.vis_re, other.vis_im, other.B, other.V, nb)
        ha = im.pipe_host(small.vis_re, small.vis_im, small.B, small.V, nb)
        torch.cuda.synchronize()
    tol = 1e-5
    assert np.abs(ra.cpu().numpy().reshape(u, u) - ref_a).max() <= tol
    assert np.abs(rb.cpu().numpy().reshape(u, u) - ref_b).max() <= tol
    assert np.abs(ha - ref_a).max() <= tol
    assert np.abs(hb - ref_b).max() <= tol


def test_sequence_matches_triples(cuda):
    import torch
    snap = synthetic.config_tiny(n_snap=5, transient_snapshot=3)
    n, nb, t = snap.image_size, snap.num_baselines, snap.unit_size
    u = n // t
    d = to_dev(snap, cuda)
    seq = torch.zeros(3 * u * u, device=cuda)
    with fip.Imager(n, nb, snap.cell_size, t) as im:
        im.image_sequence(d["vis_re"], d["vis_im"], d["B"], d["V"], [nb] * 5, nb, seq)
        torch.cuda.synchronize()
    seq = seq.cpu().numpy().reshape(3, u, u)
    for k in range(3):
        sub = synthetic.SnapshotSet(
            vis_re=snap.vis_re[k * nb:(k + 3) * nb], vis_im=snap.vis_im[k * nb:(k + 3) * nb],
            B=snap.B[2 * k * nb:2 * (k + 3) * nb], V=snap.V[9 * k:9 * (k + 3)],
            num_baselines=nb, num_snapshots=3, image_size=n, cell_size=snap.cell_size,
            unit_size=t, frequency_hz=snap.frequency_hz)
        res, _, _ = run(sub, cuda)
        assert np.abs(seq[k] - res).max() <= 1e-6


# ---------------------------------------------------------------- edge cases

def test_identical_snapshots_give_unit_tlisi(cuda):
    snap = synthetic.config_tiny()
    nb = snap.num_baselines
    for a in (snap.vis_re, snap.vis_im):
        a[nb:2 * nb] = a[:nb]
        a[2 * nb:] = a[:nb]
    snap.B[2 * nb:4 * nb] = snap.B[:2 * nb]
    snap.B[4 * nb:] = snap.B[:2 * nb]
    snap.V[9:18] = snap.V[:9]
    snap.V[18:] = snap.V[:9]
    res, _, _ = run(snap, cuda)
    assert np.abs(res - 1.0).max() <= 1e-6


@pytest.mark.parametrize("storage,tol", [(fip.STORE_F16, 1e-3), (fip.STORE_BF16, 8e-3)])
def test_reduced_storage_block_scales_at_extreme_blocks(cuda, storage, tol):
    """Reduced storage keeps one power-of-two scale per 1,024 visibilities:
    a block of zeros (the smallest scale), a block 1e12 brighter and one
    1e-12 fainter than the rest, and a partial last block (2,145 samples
    per snapshot here) image as with FP32 storage within the storage's
    rounding, in the precision form."""
    snap = synthetic.config_small(n_ant=66, transient_snapshot=2)
    nb = snap.num_baselines
    assert nb % 1024 != 0 and nb > 2048
    for k in range(3):
        v = slice(k * nb, (k + 1) * nb)
        for arr in (snap.vis_re, snap.vis_im):
            a = arr[v]
            a[:1024] = 0.0
            a[1024:2048] *= 1e12 if k != 1 else 1e-12
    want, wimg, _ = run(snap, cuda, form=fip.FORM_PRECISE, vis_storage=fip.STORE_F32)
    got, gimg, _ = run(snap, cuda, form=fip.FORM_PRECISE, vis_storage=storage)
    assert np.isfinite(gimg).all()
    for k in range(3):
        assert relrms(gimg[k], wimg[k]) <= tol
    both = np.isfinite(want) & np.isfinite(got)
    assert np.array_equal(np.isfinite(want), np.isfinite(got))
    assert np.abs(got - want)[both].max() <= 50 * tol


def test_zero_visibilities_give_nan_like_reference(cuda):
    snap = synthetic.config_tiny()
    snap.vis_re[:] = 0
    snap.vis_im[:] = 0
    res, imgs, mx = run(snap, cuda)
    assert np.all(mx == 0) and np.all(imgs == 0)
    assert np.all(np.isnan(res))


def test_flagged_zero_padded_baselines(cuda):
    snap = synthetic.config_tiny(flag_fraction_max=0.3, transient_snapshot=2, seed=9)
    res, imgs, _ = run(snap, cuda, form=fip.FORM_PRECISE)
    r64, i64, _ = oracle.fipipe(snap, "f64", want_images=True)
    assert np.abs(res - r64).max() <= 1e-4
    for k in range(3):
        assert relrms(imgs[k], i64[k]) <= 3e-5


def test_single_baseline_and_ragged_tiles(cuda):
    """One baseline: the plane fit is degenerate (V22 = 0, the reference's
    coordschange divides by zero and splats nothing), which the gather flags
    as outside its domain; the result still equals the oracle's."""
    snap = synthetic.config_tiny(n_ant=2, unit_size=24, transient_snapshot=None)
    assert snap.num_baselines == 1
    res, imgs, _ = run(snap, cuda, check=False, form=fip.FORM_PRECISE)
    r64, i64, _ = oracle.fipipe(snap, "f64", want_images=True)
    assert res.shape == (5, 5)
    assert np.allclose(res, r64, atol=1e-4, equal_nan=True)


def test_invalid_sizes_raise(cuda):
    with pytest.raises(fip.FipError):
        fip.Imager(102, 10, 1e-3, 16)
    with fip.Imager(64, 10, 1e-3, 16) as im:
        import torch
        z = torch.zeros(1000, device=cuda)
        with pytest.raises(fip.FipError):
            im.image_snapshot(z, z, z, z, 11, z)
        # The host-buffer path checks nb against the imager's capacity before
        # it stages anything into its pinned block.
        h = np.zeros(3 * 2 * 11, np.float32)
        for bad in (11, 0):
            with pytest.raises(fip.FipError):
                im.pipe_host(h, h, h, np.zeros(27, np.float32), bad)


def test_profiling_and_launch_count(cuda, tiny):
    import torch
    d = to_dev(tiny, cuda)
    u = tiny.image_size // tiny.unit_size
    out = torch.zeros(u * u, device=cuda)
    with fip.Imager(tiny.image_size, tiny.num_baselines, tiny.cell_size, tiny.unit_size) as im:
        im.set_profiling(True)
        before = im.kernel_launches
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], tiny.num_baselines, out)
        st = im.stage_times()
        assert im.kernel_launches - before >= 3 * 8 + 1
        for k in ("bin", "grid", "fft_rows", "targets", "reproject", "trigger"):
            assert st[k][1] >= 1 and st[k][0] > 0


@pytest.mark.parametrize("vpt,split,direct,ctas", [(8, 0, 0, 3), (16, 0, 0, 2), (8, 1, 0, 1),
                                                   (16, 1, 0, 4), (8, 0, 1, 2), (16, 0, 1, 3),
                                                   (16, 0, 2, 4), (8, 0, 2, 1)])
def test_every_launch_shape_gives_the_same_results(cuda, small, vpt, split, direct, ctas):
    """Transform values per thread, split/joint transform and gridder CTAs per SM
    change rounding only."""
    import torch
    n, nb, t = small.image_size, small.num_baselines, small.unit_size
    u = n // t
    d = to_dev(small, cuda)
    ref, got = torch.zeros(u * u, device=cuda), torch.zeros(u * u, device=cuda)
    with fip.Imager(n, nb, small.cell_size, t) as im:
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, ref)
        im.set_tuning(vpt, split, ctas, direct)
        assert im.tuning() == {"fft_values_per_thread": vpt, "fft_split": split,
                               "fft_direct": direct, "grid_ctas_per_sm": ctas}
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, got)
        torch.cuda.synchronize()
    assert np.abs(got.cpu().numpy() - ref.cpu().numpy()).max() <= 1e-5


@pytest.mark.parametrize("direct", [1, 2])
def test_row_pass_band_copy_at_reference_shape(cuda, direct):
    """The row pass's first pass reading global memory (1) or a band copy brought
    in by bulk tensor copies (2) gives the staged form's images up to rounding,
    at 4096^2 (a persistent launch over 2048 row pairs)."""
    import torch
    snap = synthetic.config_reference(transient_snapshot=2)
    n, nb, t = snap.image_size, snap.num_baselines, snap.unit_size
    d = to_dev(snap, cuda)
    with fip.Imager(n, nb, snap.cell_size, t) as im:
        imgs = []
        for dr in (0, direct):
            im.set_tuning(16, 0, 4, dr)
            assert im.tuning()["fft_direct"] == dr
            img = torch.zeros(n * n, device=cuda)
            mx = torch.zeros(1, device=cuda)
            im.image_snapshot(d["vis_re"][:nb], d["vis_im"][:nb], d["B"][:2 * nb], d["V"][:9], nb,
                              img, mx)
            torch.cuda.synchronize()
            imgs.append(img.cpu().numpy())
    assert relrms(imgs[1], imgs[0]) <= 1e-6


@pytest.mark.parametrize("form", ["plain", "precise", "precise_f32"])
def test_autotune_keeps_results(cuda, small, form):
    """The autotuner only picks launch shapes: results stay within rounding."""
    import torch
    kw = ({} if form == "plain" else
          dict(form=fip.FORM_PRECISE,
               vis_storage=fip.STORE_F32 if form == "precise_f32" else fip.STORE_F16))
    n, nb, t = small.image_size, small.num_baselines, small.unit_size
    u = n // t
    d = to_dev(small, cuda)
    before, after = torch.zeros(u * u, device=cuda), torch.zeros(u * u, device=cuda)
    with fip.Imager(n, nb, small.cell_size, t, **kw) as im:
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, before)
        choice = im.autotune(d["vis_re"], d["vis_im"], d["B"], d["V"], nb)
        assert choice["fft_values_per_thread"] in (8, 16)
        # Two-limb compensated sums (FP32 storage) fit 3 gridder CTAs per SM,
        # one-limb sums (plain form, FP16/BF16 storage) 4.
        assert 1 <= choice["grid_ctas_per_sm"] <= (3 if form == "precise_f32" else 4)
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, after)
        torch.cuda.synchronize()
    assert np.abs(after.cpu().numpy() - before.cpu().numpy()).max() <= 1e-5


# ---------------------------------------------------------------- preprocessing

def test_plane_projection_vs_oracle(cuda):
    import torch
    snap = synthetic.config_small()
    rows = snap.num_baselines
    freqs = np.array([130e6, 140e6, 150e6], np.float32)
    uvw = snap.uvw_m[0].reshape(-1).astype(np.float32)
    B = torch.zeros(rows * 3 * 2, device=cuda)
    V = torch.zeros(9, device=cuda)
    fip.plane_project(torch.tensor(uvw, device=cuda), torch.tensor(freqs, device=cuda), rows, 3,
                      B, V)
    torch.cuda.synchronize()
    Bo, Vo = oracle.plane_fit(uvw.reshape(-1, 3), freqs)
    assert np.allclose(V.cpu().numpy().reshape(3, 3), Vo, atol=1e-6)
    assert np.allclose(B.cpu().numpy().reshape(-1, 2), Bo, rtol=1e-5, atol=1e-3)


def test_collapse_vs_oracle(cuda):
    import torch
    rng = np.random.default_rng(3)
    ns = 10000
    arrs = [rng.standard_normal(ns).astype(np.float32) for _ in range(4)]
    f0 = (rng.random(ns) < 0.3).astype(np.uint8)
    f3 = (rng.random(ns) < 0.3).astype(np.uint8)
    w0 = rng.random(ns).astype(np.float32)
    w3 = rng.random(ns).astype(np.float32)
    t = lambda a: torch.tensor(a, device=cuda)
    o_re = torch.zeros(ns, device=cuda)
    o_im = torch.zeros(ns, device=cuda)
    fip.collapse_visibilities(*(t(a) for a in arrs), t(f0), t(f3), t(w0), t(w3), o_re, o_im, ns)
    torch.cuda.synchronize()
    w_re, w_im = oracle.collapse(*arrs, f0, f3, w0, w3)
    assert np.allclose(o_re.cpu().numpy(), w_re, rtol=1e-6, atol=1e-6)
    assert np.allclose(o_im.cpu().numpy(), w_im, rtol=1e-6, atol=1e-6)


# ---------------------------------------------------------------- command line

@pytest.mark.parametrize("with_freq", [True, False])
def test_cli_end_to_end(cuda, tiny, tmp_path, with_freq):
    nb, n = tiny.num_baselines, tiny.image_size
    p = {k: str(tmp_path / f"{k}.fits") for k in ("vr", "vi", "B", "V")}
    fits.write_image(p["vr"], tiny.vis_re[:, None])
    fits.write_image(p["vi"], tiny.vis_im[:, None])
    fits.write_image(p["B"], tiny.B.reshape(-1, 2))
    fits.write_image(p["V"], tiny.V.reshape(-1, 3))
    out = str(tmp_path / "out.fits")
    args = [fip.CLI_PATH, p["vr"], p["vi"], p["B"], p["V"], str(n), str(nb)]
    if with_freq:
        args.append(str(tiny.frequency_hz))
    args += [repr(tiny.cell_size), "3", str(tiny.unit_size), out]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = fits.read_image(out)
    want = fip.FIpipe(tiny.vis_re, tiny.vis_im, tiny.B, tiny.V, nb, n, 3, tiny.cell_size,
                      tiny.unit_size)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-6
