"""Multi-process (world size 2, gloo, CPU) tests of the per-beam sharding and
the max-over-ranks timing reduction used by bench.py."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fastimagingpipe_b200 import multi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        beams = multi.beams_for_rank(5, world, rank)
        t = multi.max_over_ranks(1.0 + rank)
        s = multi.sum_over_ranks(len(beams))
        q.put((rank, beams, t, s))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        rank, beams, t, s = q.get(timeout=120)
        got[rank] = (beams, t, s)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0][0] == [0, 2, 4] and got[1][0] == [1, 3]
    assert got[0][1] == got[1][1] == 2.0
    assert got[0][2] == got[1][2] == 5


def test_single_process_fallbacks():
    assert multi.max_over_ranks(3.5) == 3.5
    assert multi.whole_job_throughput([3, 3], [1.0, 2.0]) == 3.0
    with pytest.raises(ValueError):
        multi.beams_for_rank(4, 2, 2)


def _cpu_image(k, image, image_max, n=32):
    """A seeded stand-in image for snapshot k (the exchange logic is what is
    tested here; the imaging itself is the GPU tests')."""
    import numpy as np
    rng = np.random.default_rng(100 + k)
    img = rng.random(n * n).astype(np.float32)
    img[(k * 37) % (n * n)] += 4.0
    image.copy_(torch.from_numpy(img))
    image_max.fill_(float(img.max()))


def _cpu_window(images, maxima, count, results, n=32, t=8):
    import numpy as np
    import oracle
    x = images.numpy().astype(np.float64).reshape(count, n, n)
    m = maxima.numpy().astype(np.float64)
    for i in range(count - 2):
        results[i].copy_(torch.from_numpy(
            oracle.tlisi(x[i], x[i + 1], x[i + 2], m[i:i + 3], t).astype(np.float32).ravel()))


def _range_worker(rank, world, port, n_snap, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = multi.image_range_sharded(n_snap, 32, 8, _cpu_image, _cpu_window)
        q.put((rank, {k: v.numpy() for k, v in out.items()}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_snap", [(2, 7), (3, 9)])
def test_snapshot_range_sharding_equals_one_run(world, n_snap):
    """Each rank images its contiguous range and receives the previous range's
    last two images: the union of the ranks' tLISI matrices is the single-run
    sliding window, boundary triples included."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_range_worker, args=(r, world, port, n_snap, q))
             for r in range(world)]
    for p in procs:
        p.start()
    merged = {}
    for _ in procs:
        rank, out = q.get(timeout=180)
        assert not set(out) & set(merged)
        merged.update(out)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one = multi.image_range_sharded(n_snap, 32, 8, _cpu_image, _cpu_window)
    assert sorted(merged) == sorted(one) == list(range(2, n_snap))
    for k in one:
        assert np.array_equal(merged[k], one[k].numpy())


def test_snapshot_ranges():
    assert [list(multi.snapshot_range(10, 3, r)) for r in range(3)] == [[0, 1, 2, 3], [4, 5, 6],
                                                                        [7, 8, 9]]
    with pytest.raises(ValueError):
        multi.snapshot_range(4, 2, 2)
    with pytest.raises(ValueError):
        multi.image_range_sharded(1, 32, 8, _cpu_image, _cpu_window)
