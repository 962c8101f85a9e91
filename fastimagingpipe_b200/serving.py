"""Open-loop Poisson load for the multi-beam server (the serving
configuration: several beams, snapshots arriving as independent Poisson
processes, latency measured per request from submit to result)."""
from __future__ import annotations

import threading
import time
from typing import Dict, List, Sequence

import numpy as np

from . import FipError, Server
from .synthetic import SnapshotSet


def poisson_arrivals(rates: Sequence[float], duration_s: float, seed: int = 0):
    """Merged arrival schedule [(t, beam)] of independent Poisson streams."""
    rng = np.random.default_rng(seed)
    events = []
    for beam, lam in enumerate(rates):
        t = rng.exponential(1.0 / lam)
        while t < duration_s:
            events.append((t, beam))
            t += rng.exponential(1.0 / lam)
    events.sort()
    return events


def run_poisson(server: Server, beam_ids: Sequence[int], data: Sequence[SnapshotSet],
                rates: Sequence[float], duration_s: float, seed: int = 0) -> Dict:
    """Submits each beam's snapshots (cycling through its SnapshotSet) at
    Poisson times for `duration_s`, waits for all results and reports
    throughput and latency percentiles (per beam and overall)."""
    events = poisson_arrivals(rates, duration_s, seed)
    pending: List[tuple] = []
    refused = 0
    counters = [0] * len(beam_ids)
    lock = threading.Lock()
    results: List[Dict] = []

    def waiter():
        while True:
            with lock:
                item = pending.pop(0) if pending else None
                finished = item is None and done_submitting.is_set()
            if item is None:
                if finished:
                    return
                time.sleep(0.0002)
                continue
            r = server.wait(item[0])
            r["beam_index"] = item[1]
            results.append(r)

    done_submitting = threading.Event()
    th = threading.Thread(target=waiter, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for t, b in events:
        now = time.perf_counter() - t0
        if t > now:
            time.sleep(t - now)
        snap = data[b]
        k = counters[b] % snap.num_snapshots
        counters[b] += 1
        nb = snap.num_baselines
        try:
            rid = server.submit(beam_ids[b], snap.vis_re[k * nb:(k + 1) * nb],
                                snap.vis_im[k * nb:(k + 1) * nb],
                                snap.B[2 * k * nb:2 * (k + 1) * nb], snap.V[9 * k:9 * k + 9], nb)
        except FipError:
            refused += 1
            continue
        with lock:
            pending.append((rid, b))
    done_submitting.set()
    th.join()
    elapsed = time.perf_counter() - t0
    lat = np.array([r["latency_ms"] for r in results])
    per_beam = {}
    for b in range(len(beam_ids)):
        lb = np.array([r["latency_ms"] for r in results if r["beam_index"] == b])
        if lb.size:
            per_beam[b] = {"completed": int(lb.size), "p50_ms": float(np.percentile(lb, 50)),
                           "p99_ms": float(np.percentile(lb, 99))}
    return {"completed": len(results), "refused": refused, "elapsed_s": elapsed,
            "throughput": len(results) / elapsed,
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
            "per_beam": per_beam}
