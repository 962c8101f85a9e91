"""GPU tests of the trigger's load paths.

Plain-form sliding-window triggers (fip_trigger_window, batches) stream every
tile's slices through registers, each image read once (default), or read each
triple's three images; both reduce in k_trigger's lane and shuffle order, so
the tLISI must be identical bit for bit, and equal to one fip_trigger call
per triple.  Single triples are also checked against the oracle's FP64
trigger (FIPkernels.cu:806-851) within the FP32 rounding of the sums.
"""
import numpy as np
import pytest

import fastimagingpipe_b200 as fip
import oracle

pytestmark = pytest.mark.gpu


def images(n, count, seed, cuda):
    """Sky-like images: positive noise with sources, zero patches (the clamp of
    I2 and the NaN-ratio case) and negative pixels."""
    import torch
    g = torch.Generator(device=cuda).manual_seed(seed)
    x = torch.rand(count, n, n, device=cuda, generator=g) * 0.2
    x[:, n // 3:n // 3 + 24, n // 5:n // 5 + 40] = 0.0
    x[:, ::97, ::89] += 5.0
    x[:, 7::131, ::53] -= 0.3
    mx = torch.clamp(x.reshape(count, -1).max(dim=1).values, min=0.0)
    return x.contiguous(), mx.contiguous()


def bits(t):
    return t.cpu().numpy().view(np.int32)


def run_both(fn):
    prev = fip.set_trigger_streaming(True)
    try:
        a = fn()
        fip.set_trigger_streaming(False)
        b = fn()
    finally:
        fip.set_trigger_streaming(prev)
    return a, b


@pytest.mark.parametrize("form", [fip.FORM_PLAIN, fip.FORM_PRECISE])
@pytest.mark.parametrize("n,t", [(256, 8), (512, 16), (480, 24), (1024, 32), (1000, 16),
                                 (256, 4)])
def test_triple_vs_oracle(cuda, n, t, form):
    import torch
    x, mx = images(n, 3, 11 + n + t, cuda)
    u = n // t
    out = torch.full((u * u,), -7.0, device=cuda)
    with fip.Imager(n, 16, 1e-5, t, form=form) as im:
        im.trigger(x[0], x[1], x[2], mx, out)
        torch.cuda.synchronize()
    host = x.cpu().numpy().astype(np.float64)
    want = oracle.tlisi(host[0], host[1], host[2], mx.cpu().numpy().astype(np.float64), t)
    got = out.cpu().numpy().reshape(u, u)
    ok = np.isfinite(want)
    assert np.array_equal(ok, np.isfinite(got))
    assert np.abs(got[ok] - want[ok]).max() <= 1e-5


@pytest.mark.parametrize("form", [fip.FORM_PLAIN, fip.FORM_PRECISE])
@pytest.mark.parametrize("n,t,count", [(512, 32, 3), (512, 16, 9), (1024, 32, 20),
                                       (256, 24, 5), (256, 12, 6), (256, 8, 66),
                                       (4096, 32, 18), (1000, 16, 11), (256, 36, 7),
                                       (2048, 4, 4)])
def test_window_streamed_equals_per_triple(cuda, n, t, count, form):
    import torch
    x, mx = images(n, count, 5 * count + t, cuda)
    u = n // t

    def run():
        out = torch.full(((count - 2) * u * u,), -7.0, device=cuda)
        with fip.Imager(n, 16, 1e-5, t, form=form) as im:
            im.trigger_window(x, mx, count, out)
            torch.cuda.synchronize()
        return out

    a, b = run_both(run)
    assert np.array_equal(bits(a), bits(b))
    # Triple k of the window is fip_trigger on images k, k+1, k+2.
    with fip.Imager(n, 16, 1e-5, t, form=form) as im:
        for k in range(count - 2):
            one = torch.zeros(u * u, device=cuda)
            im.trigger(x[k], x[k + 1], x[k + 2], mx[k:k + 3].contiguous(), one)
            torch.cuda.synchronize()
            assert np.array_equal(bits(one), bits(a[k * u * u:(k + 1) * u * u]))


def test_window_argument_errors(cuda):
    import torch
    x, mx = images(256, 3, 1, cuda)
    out = torch.zeros(64, device=cuda)
    with fip.Imager(256, 16, 1e-5, 32) as im:
        with pytest.raises(fip.FipError):
            im.trigger_window(x, mx, 2, out)
    with fip.Imager(256, 16, 1e-5, 0) as im:
        with pytest.raises(fip.FipError):
            im.trigger_window(x, mx, 3, out)
