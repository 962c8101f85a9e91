"""GPU tests of the batching form (fip_batch): one persistent gridding launch
and one batched transform per call, replayed as a CUDA graph, against the
per-snapshot path and the FP64 oracle.

Tolerances: batch vs the per-snapshot path 1e-5 absolute in tLISI (the same
kernels; float-atomic gridding sums may round in another order); precision
form vs FP64 1e-4 absolute (the parity bar of the precision form).
"""
from types import SimpleNamespace

import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import synthetic
import oracle

pytestmark = pytest.mark.gpu


def mfs(n_snap=6, seed=5):
    # 64 antennas, 2 channels, 0-30 % flagged: uneven nb per snapshot.
    return synthetic.config_batching(512, n_snap=n_snap, n_chan=2, n_ant=64, radius_m=1500.0,
                                     core_fraction=0.0, transient_snapshot=3, seed=seed)


def dev(snaps, cuda):
    import torch
    return [{k: torch.tensor(getattr(s, k), device=cuda) for k in ("vis_re", "vis_im", "B", "V")}
            for s in snaps]


def per_snapshot(snaps, d, cuda, **kw):
    """Sliding-window tLISI through the per-snapshot entry points."""
    import torch
    s0 = snaps[0]
    n, t = s0.image_size, s0.unit_size
    u = n // t
    nbmax = max(s.nb for s in snaps)
    imgs = torch.zeros((len(snaps), n * n), device=cuda)
    mx = torch.zeros(len(snaps), device=cuda)
    out = []
    with fip.Imager(n, nbmax, s0.cell_size, t, **kw) as im:
        for k, s in enumerate(snaps):
            im.image_snapshot(d[k]["vis_re"], d[k]["vis_im"], d[k]["B"], d[k]["V"], s.nb,
                              imgs[k], mx[k:])
        for k in range(2, len(snaps)):
            r = torch.zeros(u * u, device=cuda)
            im.trigger(imgs[k - 2], imgs[k - 1], imgs[k], mx[k - 2:], r)
            out.append(r)
        torch.cuda.synchronize()
    return np.stack([r.cpu().numpy().reshape(u, u) for r in out])


def batched(snaps, d, cuda, calls, **kw):
    import torch
    s0 = snaps[0]
    n, t = s0.image_size, s0.unit_size
    u = n // t
    nbmax = max(s.nb for s in snaps)
    res = torch.zeros((len(snaps), u * u), device=cuda)
    got = 0
    with fip.Batch(n, nbmax, s0.cell_size, t, max(calls), **kw) as b:
        k = 0
        for c in calls:
            part = d[k:k + c]
            got += b.image([p["vis_re"] for p in part], [p["vis_im"] for p in part],
                           [p["B"] for p in part], [p["V"] for p in part],
                           [s.nb for s in snaps[k:k + c]], res[got:])
            k += c
        torch.cuda.synchronize()
        launches = b.kernel_launches
    assert got == len(snaps) - 2
    return res[:got].cpu().numpy().reshape(got, u, u), launches


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)])
def test_batch_matches_per_snapshot_path(cuda, kw):
    snaps = mfs()
    d = dev(snaps, cuda)
    ref = per_snapshot(snaps, d, cuda, **kw)
    got, launches = batched(snaps, d, cuda, [6], **kw)
    assert launches > 0
    assert np.abs(got - ref).max() <= 1e-5


def test_batch_carries_the_sequence_across_calls(cuda):
    snaps = mfs()
    d = dev(snaps, cuda)
    one, _ = batched(snaps, d, cuda, [6])
    split, _ = batched(snaps, d, cuda, [2, 1, 3])
    assert np.abs(one - split).max() <= 1e-5


def test_batch_graph_replay_with_new_inputs(cuda):
    """The executable graph is re-used across calls of one shape: results must
    follow the new inputs, not the captured ones."""
    import torch
    a, b2 = mfs(seed=5), mfs(seed=9)
    da, db = dev(a, cuda), dev(b2, cuda)
    ref_b = per_snapshot(b2, db, cuda)
    s0 = a[0]
    u = s0.image_size // s0.unit_size
    nbmax = max(s.nb for s in a + b2)
    with fip.Batch(s0.image_size, nbmax, s0.cell_size, s0.unit_size, 6) as b:
        res = torch.zeros((4, u * u), device=cuda)
        for snaps, d in ((a, da), (b2, db)):
            b.reset()
            b.image([p["vis_re"] for p in d], [p["vis_im"] for p in d], [p["B"] for p in d],
                    [p["V"] for p in d], [s.nb for s in snaps], res)
        torch.cuda.synchronize()
    assert np.abs(res.cpu().numpy().reshape(4, u, u) - ref_b).max() <= 1e-5


def test_batch_precision_form_vs_fp64(cuda):
    small = synthetic.config_small(transient_snapshot=2)
    nb = small.num_baselines
    import torch
    d = [{"vis_re": torch.tensor(small.vis_re[k * nb:(k + 1) * nb], device=cuda),
          "vis_im": torch.tensor(small.vis_im[k * nb:(k + 1) * nb], device=cuda),
          "B": torch.tensor(small.B[2 * k * nb:2 * (k + 1) * nb], device=cuda),
          "V": torch.tensor(small.V[9 * k:9 * (k + 1)], device=cuda)} for k in range(3)]
    u = small.image_size // small.unit_size
    res = torch.zeros(u * u, device=cuda)
    with fip.Batch(small.image_size, nb, small.cell_size, small.unit_size, 3,
                   form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16) as b:
        tuning = b.autotune([p["vis_re"] for p in d], [p["vis_im"] for p in d],
                            [p["B"] for p in d], [p["V"] for p in d], [nb] * 3)
        assert tuning["fft_values_per_thread"] in (8, 16)
        assert b.image([p["vis_re"] for p in d], [p["vis_im"] for p in d], [p["B"] for p in d],
                       [p["V"] for p in d], [nb] * 3, res) == 1
        torch.cuda.synchronize()
    r64, _, _ = oracle.fipipe(small, "f64")
    assert np.abs(res.cpu().numpy().reshape(u, u) - r64).max() <= 1e-4


def test_batch_rejects_bad_arguments(cuda):
    import torch
    with pytest.raises(fip.FipError):
        fip.Batch(102, 10, 1e-3, 17, 4)  # not a multiple of 4
    with pytest.raises(fip.FipError):
        fip.Batch(64, 10, 1e-3, 16, 65)  # above the batch limit
    z = torch.zeros(64, device=cuda)
    with fip.Batch(64, 10, 1e-3, 16, 2) as b:
        with pytest.raises(fip.FipError):
            b.image([z] * 3, [z] * 3, [z] * 3, [z] * 3, [5] * 3, z)  # count > max_snapshots
        with pytest.raises(fip.FipError):
            b.image([z], [z], [z], [z], [11], z)  # nb > max_baselines


def mfs_n(n, n_snap, seed):
    return synthetic.config_batching(n, n_snap=n_snap, n_chan=2, n_ant=64, radius_m=1500.0,
                                     core_fraction=0.0, transient_snapshot=2, seed=seed)


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)])
@pytest.mark.parametrize("calls", [[11], [4, 7]])
def test_mixed_sizes_in_one_batch(cuda, kw, calls):
    """Two sequences of different image sizes (512^2 and 256^2, the cell scaled
    for the same field) imaged together: one persistent gridding launch per
    call over both; each sequence's sliding-window tLISI must equal its
    per-snapshot path's."""
    import torch
    big, small = mfs_n(512, 6, 5), mfs_n(256, 5, 7)
    db, ds = dev(big, cuda), dev(small, cuda)
    ref = [per_snapshot(big, db, cuda, **kw), per_snapshot(small, ds, cuda, **kw)]
    # Interleaved call order: 512, 256, 512, 256, ...
    order = []
    ib = is_ = 0
    while ib < len(big) or is_ < len(small):
        if ib < len(big):
            order.append((0, ib))
            ib += 1
        if is_ < len(small):
            order.append((1, is_))
            is_ += 1
    seqs = [big, small]
    devs = [db, ds]
    spec = [(s[0].image_size, max(x.nb for x in s), s[0].cell_size, s[0].unit_size) for s in seqs]
    us = [x[0] // x[3] for x in spec]
    res = [torch.zeros((len(s), u * u), device=cuda) for s, u in zip(seqs, us)]
    got = [0, 0]
    with fip.Batch.of_sequences(spec, 6, **kw) as b:
        tunes = b.autotune_sequences([c for c, _ in order[:6]],
                                     *[[devs[c][i][key] for c, i in order[:6]]
                                       for key in ("vis_re", "vis_im", "B", "V")],
                                     [seqs[c][i].nb for c, i in order[:6]])
        assert len(tunes) == 2
        k = 0
        for n_call in calls:
            part = order[k:k + n_call]
            k += n_call
            counts = b.image_sequences(
                [c for c, _ in part],
                *[[devs[c][i][key] for c, i in part] for key in ("vis_re", "vis_im", "B", "V")],
                [seqs[c][i].nb for c, i in part],
                [res[0][got[0]:], res[1][got[1]:]])
            got = [g + n for g, n in zip(got, counts)]
        torch.cuda.synchronize()
        b.check()
        assert b.kernel_launches > 0
    assert got == [len(big) - 2, len(small) - 2]
    for c in range(2):
        out = res[c][:got[c]].cpu().numpy().reshape(got[c], us[c], us[c])
        assert np.abs(out - ref[c]).max() <= 1e-5


def test_sequences_reject_bad_arguments(cuda):
    import torch
    spec = [(64, 10, 1e-3, 16), (128, 10, 5e-4, 16)]
    with pytest.raises(fip.FipError):
        fip.Batch.of_sequences(spec * 5, 2)  # more than 8 sequences
    z = torch.zeros(64, device=cuda)
    with fip.Batch.of_sequences(spec, 2) as b:
        with pytest.raises(fip.FipError):
            b.image_sequences([2], [z], [z], [z], [z], [5], [z, z])  # no such sequence
        with pytest.raises(fip.FipError):
            b.image_sequences([1, 1, 1], [z] * 3, [z] * 3, [z] * 3, [z] * 3, [5] * 3,
                              [z, z])  # more than max_snapshots of one sequence
    lib = fip.lib()
    import ctypes
    cfgs = (fip.ImagerConfig * 2)(fip.ImagerConfig(64, 10, 16, 1e-3, fip.FORM_PLAIN, 0, 0, 0),
                                  fip.ImagerConfig(128, 10, 16, 5e-4, fip.FORM_PRECISE, 0, 0, 0))
    h = ctypes.c_void_p()
    assert lib.fip_batch_create_sequences(ctypes.byref(h), ctypes.cast(cfgs, ctypes.c_void_p),
                                          2, 2) == 1  # forms differ


@pytest.mark.parametrize("kw", [{}, dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)])
def test_batch_of_cufft_and_pruned_sizes(cuda, kw):
    """A 100^2 sequence (grid side 150: a batched cuFFT C2R plan) and a 128^2
    sequence (band-pruned transform) imaged together, over calls of two
    sizes (two cuFFT plans): each sequence's tLISI equals its per-snapshot
    path's."""
    import torch
    odd = [synthetic.config_tiny(image_size=100, cell_size=1.5e-4, unit_size=20,
                                 transient_snapshot=2, n_snap=5, seed=31)]
    pow2 = [synthetic.config_tiny(transient_snapshot=2, n_snap=5, seed=32)]
    seqs = []
    for s in (odd[0], pow2[0]):
        nb = s.num_baselines
        seqs.append([SimpleNamespace(vis_re=s.vis_re[k * nb:(k + 1) * nb],
                                     vis_im=s.vis_im[k * nb:(k + 1) * nb],
                                     B=s.B[2 * k * nb:2 * (k + 1) * nb], V=s.V[9 * k:9 * k + 9],
                                     nb=nb, image_size=s.image_size, unit_size=s.unit_size,
                                     cell_size=s.cell_size) for k in range(5)])
    devs = [dev(x, cuda) for x in seqs]
    ref = [per_snapshot(x, d, cuda, **kw) for x, d in zip(seqs, devs)]
    spec = [(x[0].image_size, x[0].nb, x[0].cell_size, x[0].unit_size) for x in seqs]
    us = [x[0] // x[3] for x in spec]
    res = [torch.zeros((5, u * u), device=cuda) for u in us]
    order = [(c, k) for k in range(5) for c in range(2)]
    got = [0, 0]
    with fip.Batch.of_sequences(spec, 5, **kw) as b:
        for part in (order[:4], order[4:]):
            counts = b.image_sequences(
                [c for c, _ in part],
                *[[devs[c][k][key] for c, k in part] for key in ("vis_re", "vis_im", "B", "V")],
                [seqs[c][k].nb for c, k in part], [res[0][got[0]:], res[1][got[1]:]])
            got = [g + n for g, n in zip(got, counts)]
        torch.cuda.synchronize()
        b.check()
    assert got == [3, 3]
    for c in range(2):
        out = res[c][:3].cpu().numpy().reshape(3, us[c], us[c])
        assert np.abs(out - ref[c]).max() <= 1e-5
