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
