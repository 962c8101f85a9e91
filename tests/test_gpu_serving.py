"""GPU tests of the multi-beam streaming server (fip_server).

Continuous batching must not change results: every beam's sliding-window
tLISI is the same served alone and served in a mix of beams whose requests
are merged into shared batched launches and overlap on the device
(tolerance 1e-6: only FP32 summation order may differ), and the same as the
per-snapshot imager's.
"""
import numpy as np
import pytest

import fastimagingpipe_b200 as fip
from fastimagingpipe_b200 import synthetic

pytestmark = pytest.mark.gpu

GB = 1 << 30


def beam_data(kind, seed):
    if kind == "small":
        return synthetic.config_small(n_snap=5, transient_snapshot=3, seed=seed)
    return synthetic.config_tiny(n_snap=5, transient_snapshot=3, seed=seed)


def add(sv, snap):
    return sv.add_beam(snap.image_size, snap.num_baselines, snap.cell_size, snap.unit_size)


def submit_all(sv, beam, snap):
    nb = snap.num_baselines
    return [sv.submit(beam, snap.vis_re[k * nb:(k + 1) * nb], snap.vis_im[k * nb:(k + 1) * nb],
                      snap.B[2 * k * nb:2 * (k + 1) * nb], snap.V[9 * k:9 * k + 9], nb)
            for k in range(snap.num_snapshots)]


def test_results_same_alone_and_in_the_mix(cuda):
    A = beam_data("small", 1)
    others = [beam_data("tiny", 2), beam_data("small", 3), beam_data("tiny", 4)]
    with fip.Server(20 * GB, slots=1) as sv:
        b = add(sv, A)
        alone = [sv.wait(r) for r in submit_all(sv, b, A)]
    with fip.Server(20 * GB, slots=4) as sv:
        ids = [add(sv, s) for s in [A] + others]
        nb = [s.num_baselines for s in [A] + others]
        reqs = {i: [] for i in ids}
        for k in range(5):  # interleave the beams' snapshots
            for i, s in zip(ids, [A] + others):
                n = s.num_baselines
                reqs[i].append(sv.submit(i, s.vis_re[k * n:(k + 1) * n], s.vis_im[k * n:(k + 1) * n],
                                         s.B[2 * k * n:2 * (k + 1) * n], s.V[9 * k:9 * k + 9], n))
        mixed = {i: [sv.wait(r) for r in reqs[i]] for i in ids}
        st = sv.stats()
    # 20 requests queued at once over two groups of two beams: the steps
    # merged several snapshots each.
    assert st["snapshots"] == 20 and st["steps"] < st["snapshots"]
    got = mixed[ids[0]]
    for a, m in zip(alone, got):
        assert a["seq"] == m["seq"]
        if a["tlisi"] is None:
            assert m["tlisi"] is None
        else:
            assert np.abs(a["tlisi"] - m["tlisi"]).max() <= 1e-6
    assert [r["tlisi"] is None for r in alone] == [True, True, False, False, False]
    for i in ids:
        assert [r["seq"] for r in mixed[i]] == list(range(5))
        assert all(r["latency_ms"] > 0 for r in mixed[i])
    assert nb[0] == A.num_baselines


def test_server_matches_sequence_api(cuda):
    import torch
    A = beam_data("tiny", 6)
    n, nb, t = A.image_size, A.num_baselines, A.unit_size
    u = n // t
    with fip.Server(4 * GB, slots=2) as sv:
        b = add(sv, A)
        res = [sv.wait(r) for r in submit_all(sv, b, A)]
    d = {k: torch.tensor(getattr(A, k), device=cuda) for k in ("vis_re", "vis_im", "B", "V")}
    seq = torch.zeros(3 * u * u, device=cuda)
    with fip.Imager(n, nb, A.cell_size, t) as im:
        im.image_sequence(d["vis_re"], d["vis_im"], d["B"], d["V"], [nb] * 5, nb, seq)
        torch.cuda.synchronize()
    seq = seq.cpu().numpy().reshape(3, u, u)
    for k in range(3):
        assert np.abs(res[k + 2]["tlisi"] - seq[k]).max() <= 1e-6


def test_budget_admission(cuda):
    big = synthetic.config_reference(n_snap=1)
    with fip.Server(256 * 1024 * 1024, slots=1) as sv:
        with pytest.raises(fip.FipError) as ei:
            add(sv, big)
        assert ei.value.status == 5
        assert sv.reserved_bytes == 0
        tiny = beam_data("tiny", 7)
        add(sv, tiny)
        assert 0 < sv.reserved_bytes <= 256 * 1024 * 1024


def test_queue_back_pressure(cuda):
    A = beam_data("small", 8)
    nb = A.num_baselines
    refused = 0
    with fip.Server(8 * GB, slots=1, max_queue=1) as sv:
        b = add(sv, A)
        ids = []
        for k in range(60):
            j = k % 5
            try:
                ids.append(sv.submit(b, A.vis_re[j * nb:(j + 1) * nb], A.vis_im[j * nb:(j + 1) * nb],
                                     A.B[2 * j * nb:2 * (j + 1) * nb], A.V[9 * j:9 * j + 9], nb))
            except fip.FipError as e:
                assert e.status == 6
                refused += 1
        for r in ids:
            sv.wait(r)
    assert refused > 0
