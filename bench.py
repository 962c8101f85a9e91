#!/usr/bin/env python
"""Benchmark of the snapshot imaging + tLISI trigger path on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Workload (one "step"): the reference shape -- 3 snapshots of 130,816
baselines imaged at 4096 x 4096 (grid 6144, cell 7.2722e-6 rad) and their
128 x 128 tLISI matrix (tile 32), i.e. one FIpipe call (FIPkernels.cu:554).
Inputs are seeded synthetic snapshots with the benchmark's layout, sky and
noise (fastimagingpipe_b200.synthetic.config_reference).

Prints ONE JSON line.  `value` is snapshots/s of the plain FP32 form
(reference-faithful arithmetic) with inputs resident in HBM, timed with CUDA
events around each step (L2 flushed between steps, flush untimed), summed
over the K steps, max over ranks.  `e2e` is the same metric through the
drop-in FIpipe call with host buffers (host->device copies and the result
read-back inside the timed region).  Multi-GPU: one independent beam per
rank (no data-path collective), weak scaling.

`--impl reference` runs the reference's own implementation of the path, the
unmodified FIpipe of its FIPkernels.cu recompiled for sm_100a
(oracle/_ref/libfipref.so, built by `make -C oracle ref`), on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = ("snapshots/s at 4096², 130816 bl, tLISI ≤1e-4 vs FP64 (vs plain FP32); "
          "p99 latency")
UNIT = "snapshots/s"
SNAPS_PER_STEP = 3


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(snap):
    """The FP64 CPU oracle on one full step (3 snapshots + tLISI), all host
    threads; returns (line, oracle tLISI)."""
    import oracle
    oracle.lib()
    t0 = time.perf_counter()
    res, _, _ = oracle.fipipe(snap, "f64")
    dt = time.perf_counter() - t0
    return ({"value": SNAPS_PER_STEP / dt, "unit": UNIT, "cores": oracle.num_threads(),
             "kind": "port",
             "sample": "one full step (3 snapshots at 4096^2, 130,816 baselines, tile 32) of "
                       "the FP64 OpenMP CPU restatement (oracle/fip_oracle.c)",
             "seconds": dt}, res)


def algorithmic_bytes(stage, n, nb, band, t):
    """Algorithmic bytes of one launch of a stage (the minimum it must move)."""
    k1, k2 = band
    u = n // t
    if stage == "reproject":
        return n * n * (4 + 8 + 4)      # pre + targets read, image written
    if stage == "fft_rows":
        return (k2 + 1) * n * 8 + n * n * 4
    if stage == "fft_cols":
        return (2 * k1 + 1) * (k2 + 1) * 8 + (k2 + 1) * n * 8
    if stage == "targets":
        return n * n * 8
    if stage == "trigger":
        return 3 * n * n * 4 + u * u * 4
    if stage == "grid":
        return nb * 16 + (2 * k1 + 1) * (k2 + 1) * 8
    if stage == "bin":
        return 2 * nb * 8
    return None


def _peak():
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_counters():
    """Per-stage DRAM traffic and issue counters from the committed ncu summary."""
    path = os.path.join(REPO, "profiles", "stage_counters.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def roofline_of(stage, ms, n, nb, band, t):
    """HBM roofline of one launch of a stage: algorithmic bytes / launch time
    against the measured copy bandwidth."""
    peak, src = _peak()
    alg = algorithmic_bytes(stage, n, nb, band, t)
    achieved = alg / (ms * 1e-3) / 1e9 if alg and ms > 0 else None
    prof = _profile_counters().get(stage, {})
    out = {"kernel": stage, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": (achieved / peak) if achieved else None,
           "traffic": prof.get("dram_bytes"), "peak_source": src,
           "algorithmic_bytes_per_launch": alg, "avg_launch_ms": ms}
    for k in ("issue_active_pct", "warp_instructions", "instructions_per_unit", "unit"):
        if k in prof:
            out["ncu_" + k] = prof[k]
    return out


def run_reference(args, rank):
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True}
    if rank != 0:
        return None
    from oracle import reference as ref
    if not ref.available():
        line["unavailable"] = "oracle/_ref/libfipref.so not built (make -C oracle ref)"
        return line
    from fastimagingpipe_b200 import synthetic
    snap = synthetic.config_reference()
    for _ in range(args.warmup):
        ref.fipipe(snap)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.fipipe(snap)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = SNAPS_PER_STEP * args.steps / total
    nb = snap.num_baselines
    line.update({
        "value": value, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded benchmark layout, sky and noise)",
        "config": {"workload": "FIpipe: 3 snapshots x 130,816 baselines at 4096^2, tile 32",
                   "image_size": 4096, "baselines": nb, "tile": 32, "snapshots_per_step": 3},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "unmodified reference FIpipe (FIPkernels.cu) recompiled for "
                                   "sm_100a, called with host buffers; one host thread drives "
                                   "the GPU"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "latency_ms": {"p50": 1e3 * float(np.percentile(times, 50)),
                       "p99": 1e3 * float(np.percentile(times, 99))},
    })
    return line


def run_batching(fip, synthetic, torch, dev, local, per_size=16, calls=2, distinct=4):
    """Times the batching form on configuration 4: one Batch of two sequences
    (4096^2 and 2048^2, cell scaled for one field of view), each call imaging
    `per_size` snapshots of each size interleaved (one persistent gridding launch
    for both sizes, one batched transform per size, one CUDA graph), `calls` calls
    (64 snapshots in all).  `distinct` seeded snapshots per size are generated and
    cycled (input generation on the host is the slow part)."""
    out = {}
    sizes = (4096, 2048)
    data = {}
    for n in sizes:
        snaps = synthetic.config_batching(n, n_snap=distinct, n_chan=8, seed=20 + n)
        d = [{k: torch.tensor(getattr(x, k), device=dev) for k in ("vis_re", "vis_im", "B", "V")}
             for x in snaps]
        data[n] = (snaps, d)
    total = len(sizes) * per_size * calls
    # One call: snapshot j of each size in turn.
    order = [(c, j % distinct) for j in range(per_size) for c in range(len(sizes))]
    seq = [c for c, _ in order]
    args = tuple([data[sizes[c]][1][i][key] for c, i in order]
                 for key in ("vis_re", "vis_im", "B", "V"))
    nbs = [data[sizes[c]][0][i].nb for c, i in order]
    spec = [(n, max(x.nb for x in data[n][0]), data[n][0][0].cell_size, 32) for n in sizes]
    for name, kw in (("batching_plain", {}),
                     ("batching_precise_f16", dict(form=fip.FORM_PRECISE,
                                                   vis_storage=fip.STORE_F16))):
        b = fip.Batch.of_sequences(spec, per_size, device=local, **kw)
        tunes = b.autotune_sequences(seq, *args, nbs)
        for n, tn in zip(sizes, tunes):
            out.setdefault("autotune", {})[f"{name}_{n}"] = tn
        res = [torch.zeros((per_size * calls, (n // 32) ** 2), device=dev) for n in sizes]

        def run_all():
            got = [0] * len(sizes)
            for _ in range(calls):
                counts = b.image_sequences(seq, *args, nbs, [r[g:] for r, g in zip(res, got)])
                got = [g + k for g, k in zip(got, counts)]
            return got
        b.reset()
        run_all()  # warm-up: instantiates the graph
        torch.cuda.synchronize()
        b.reset()
        l0 = b.kernel_launches
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        run_all()
        ev1.record()
        torch.cuda.synchronize()
        b.check()
        ms = ev0.elapsed_time(ev1)
        launches = b.kernel_launches - l0
        # Phase breakdown of the same calls (timing events in the graph).
        b.set_profiling(True)
        b.reset()
        run_all()
        torch.cuda.synchronize()
        ph = b.phase_times()
        b.set_profiling(False)
        out[name] = {"value": total / (ms / 1e3), "unit": UNIT, "snapshots": total,
                     "gpu_launches": launches,
                     "phases_ms_per_snapshot": {k: v / total for k, (v, c) in ph.items()},
                     "hbm_gb": b.device_bytes / 2**30,
                     "config": f"{total} snapshots x 8 channels (130-150 MHz), 0-30 % flagged, "
                               f"half 4096^2 / half 2048^2 interleaved in each call, tile 32, "
                               f"{per_size} of each size per call, one persistent gridding "
                               "launch for both sizes, CUDA graph per call"}
        b.close()
    return out


def run_batching_reference_shape(fip, torch, d, snap, dev, local, plain_value, per_call=16,
                                 calls=4):
    """The batching form on the headline shape (4096^2, 130,816 baselines, tile 32, one
    channel): the reference-shape snapshots cycled through calls of `per_call`
    snapshots; snapshots/s over `calls` calls, and the ratio to the plain form's
    device-resident value."""
    out = {}
    n, nb, t, cell = snap.image_size, snap.num_baselines, snap.unit_size, snap.cell_size
    u = n // t
    idx = [k % 3 for k in range(per_call)]
    a = ([d["vis_re"][i * nb:(i + 1) * nb] for i in idx], [d["vis_im"][i * nb:(i + 1) * nb] for i in idx],
         [d["B"][2 * i * nb:2 * (i + 1) * nb] for i in idx], [d["V"][9 * i:9 * (i + 1)] for i in idx],
         [nb] * per_call)
    res = torch.zeros((per_call, u * u), device=dev)
    stream = torch.cuda.Stream(device=dev)
    for name, kw in (("batching_plain_reference_shape", {}),
                     ("batching_precise_f16_reference_shape",
                      dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16))):
        with fip.Batch(n, nb, cell, t, per_call, device=local, **kw) as b:
            tuning = b.autotune(*a)
            with torch.cuda.stream(stream):
                b.image(*a, res, stream=stream)  # instantiates the graph
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                ev0.record(stream)
                for _ in range(calls):
                    b.image(*a, res, stream=stream)
                ev1.record(stream)
            torch.cuda.synchronize()
            v = per_call * calls / (ev0.elapsed_time(ev1) / 1e3)
            # Phase breakdown of the same calls (timing events in the graph).
            b.set_profiling(True)
            with torch.cuda.stream(stream):
                for _ in range(calls):
                    b.image(*a, res, stream=stream)
            torch.cuda.synchronize()
            ph = b.phase_times()
            b.set_profiling(False)
            out[name] = {"value": v, "unit": UNIT, "vs_plain_form": v / plain_value,
                         "autotune": tuning,
                         "phases_ms_per_snapshot": {k: ms / max(c, 1) / per_call
                                                    for k, (ms, c) in ph.items()},
                         "config": f"4096^2, 130,816 baselines, tile 32, {per_call} snapshots "
                                   f"per call, {calls} calls, CUDA graph per call"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the extra forms")
    ap.add_argument("--tuning", default=None,
                    help="pin the launch shapes VPT,SPLIT,DIRECT,CTAS instead of autotuning "
                         "(profiling runs: the autotuner's timings are not meaningful under a "
                         "profiler)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    import fastimagingpipe_b200 as fip
    from fastimagingpipe_b200 import synthetic

    dev = torch.device("cuda", local)
    snap = synthetic.config_reference(seed=1 + rank)
    n, nb, t, cell = snap.image_size, snap.num_baselines, snap.unit_size, snap.cell_size
    u = n // t
    d = {k: torch.tensor(getattr(snap, k), device=dev) for k in ("vis_re", "vis_im", "B", "V")}
    result = torch.zeros(u * u, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    im = fip.Imager(n, nb, cell, t, device=local)
    if args.tuning:
        vpt, split, direct, ctas = (int(x) for x in args.tuning.split(","))
        im.set_tuning(vpt, split, ctas, direct)
        tuning = im.tuning()
    else:
        tuning = im.autotune(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, stream=stream)

    def step():
        im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, result, stream=stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()

    # ---- device-resident timing (plain FP32 form) ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = im.kernel_launches
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()  # write 256 MB (> 126 MB L2) between steps, untimed
            starts[k].record(stream)
            step()
            ends[k].record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = im.kernel_launches - launches0
    step_ms = [starts[k].elapsed_time(ends[k]) for k in range(args.steps)]
    total_s = sum(step_ms) / 1e3
    if dist is not None:
        tt = torch.tensor([total_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_s = float(tt.item())
    value = world * SNAPS_PER_STEP * args.steps / total_s

    # ---- per-stage device times (roofline of the dominant kernel) ----
    im.set_profiling(True)
    with torch.cuda.stream(stream):
        for _ in range(max(5, min(args.steps, 20))):
            flush.zero_()
            step()
    torch.cuda.synchronize()
    stages = im.stage_times()
    im.set_profiling(False)
    band = im.band()

    # ---- end-to-end through the drop-in FIpipe (host buffers) ----
    for _ in range(2):
        fip.FIpipe(snap.vis_re, snap.vis_im, snap.B, snap.V, nb, n, 3, cell, t)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e2e_steps = max(3, min(args.steps, 50))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_res = fip.FIpipe(snap.vis_re, snap.vis_im, snap.B, snap.V, nb, n, 3, cell, t)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        tt = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_value = world * SNAPS_PER_STEP * e2e_steps / e2e_s
    clk = clocks.stop()
    h2d = SNAPS_PER_STEP * nb * (4 + 4 + 8) + SNAPS_PER_STEP * 9 * 4
    d2h = u * u * 4

    line = None
    if rank == 0:
        # The dominant kernel (largest share of the serialised stage time) and
        # its HBM roofline: algorithmic bytes per launch over the measured
        # launch time.  Its issue-side figures (from the committed ncu summary)
        # ride along, since a kernel far below the HBM roof is bound elsewhere.
        per_launch = {k: (ms / c if c else 0.0, c) for k, (ms, c) in stages.items()}
        shares = {k: per_launch[k][0] * per_launch[k][1] for k in per_launch
                  if per_launch[k][1] > 0}
        total_stage_ms = sum(shares.values())
        dom = max(shares, key=shares.get)
        roofline = roofline_of(dom, per_launch[dom][0], n, nb, band, t)
        roofline["time_share"] = shares[dom] / total_stage_ms if total_stage_ms else None
        roofline["others"] = {k: roofline_of(k, per_launch[k][0], n, nb, band, t)["frac"]
                              for k in shares if k != dom}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 512-antenna layout, 20-source sky + transient, noise 0.1)",
            "config": {"workload": "FIpipe: 3 snapshots x 130,816 baselines at 4096^2 "
                                   "(grid 6144), tile 32 -> 128x128 tLISI",
                       "image_size": n, "baselines": nb, "tile": t, "snapshots_per_step": 3,
                       "form": "plain FP32 (reference-faithful)",
                       "l2": "flushed (256 MB write) between timed steps, flush untimed",
                       "parallelism": f"{world} independent beam(s), one per GPU"},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                           "p99": float(np.percentile(step_ms, 99))},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "FIpipe (C ABI drop-in) with host numpy buffers"},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "stages_ms_per_launch": {k: v[0] for k, v in per_launch.items() if v[1]},
            "stages_note": "measured serialised (profiling run), per launch",
            "uv_band": {"max_row": band[0], "max_col": band[1], "grid": im.grid_side},
            "autotune": tuning,
        }
    # ---- extra forms (rank 0) ----
    forms = {}
    if rank == 0 and not args.no_forms:
        for name, kw in (("precise_f16", dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)),
                         ("precise_f32", dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F32))):
            im2 = fip.Imager(n, nb, cell, t, device=local, **kw)
            im2.autotune(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, stream=stream)
            res2 = torch.zeros(u * u, device=dev)
            with torch.cuda.stream(stream):
                for _ in range(3):
                    im2.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, res2,
                                    stream=stream)
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 20
            with torch.cuda.stream(stream):
                ev0.record(stream)
                for _ in range(reps):
                    im2.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, res2,
                                    stream=stream)
                ev1.record(stream)
            torch.cuda.synchronize()
            forms[name] = {"value": SNAPS_PER_STEP * reps / (ev0.elapsed_time(ev1) / 1e3),
                           "unit": UNIT, "tlisi": res2.cpu().numpy().reshape(u, u)}
            # Per-stage device times (serialised profiling calls, per launch).
            im2.set_profiling(True)
            with torch.cuda.stream(stream):
                for _ in range(5):
                    flush.zero_()
                    im2.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, res2,
                                    stream=stream)
            torch.cuda.synchronize()
            forms[name]["stages_ms_per_launch"] = {
                k: ms / c for k, (ms, c) in im2.stage_times().items() if c}
            im2.close()
        # Streaming sequence: each new snapshot yields a sliding-window tLISI.
        S = 30
        vre = torch.cat([d["vis_re"]] * 10)
        vim = torch.cat([d["vis_im"]] * 10)
        Bs = torch.cat([d["B"]] * 10)
        Vs = torch.cat([d["V"]] * 10)
        seq_res = torch.zeros((S - 2) * u * u, device=dev)
        nbs = np.full(S, nb, np.uint64)
        with torch.cuda.stream(stream):
            im.image_sequence(vre, vim, Bs, Vs, nbs, nb, seq_res, stream=stream)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            im.image_sequence(vre, vim, Bs, Vs, nbs, nb, seq_res, stream=stream)
            ev1.record(stream)
        torch.cuda.synchronize()
        forms["sequence_plain"] = {
            "value": S / (ev0.elapsed_time(ev1) / 1e3), "unit": UNIT,
            "note": "30 snapshots, sliding-window tLISI per snapshot (28 matrices)"}
        # The same sequence in the precision form (FP16 storage): the per-call
        # counterpart of the batched precision form, which also yields a
        # tLISI matrix per snapshot.
        with fip.Imager(n, nb, cell, t, form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16,
                        device=local) as imp:
            imp.autotune(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, stream=stream)
            with torch.cuda.stream(stream):
                imp.image_sequence(vre, vim, Bs, Vs, nbs, nb, seq_res, stream=stream)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                ev0.record(stream)
                imp.image_sequence(vre, vim, Bs, Vs, nbs, nb, seq_res, stream=stream)
                ev1.record(stream)
            torch.cuda.synchronize()
        forms["sequence_precise_f16"] = {
            "value": S / (ev0.elapsed_time(ev1) / 1e3), "unit": UNIT,
            "note": "30 snapshots, sliding-window tLISI per snapshot (28 matrices)"}

    # ---- batching form: 64 snapshots x 8 channels (130-150 MHz), 0-30 % flagged,
    # half at 2048^2 and half at 4096^2 (fixed field of view), tile 32 ----
    if rank == 0 and not args.no_forms:
        forms.update(run_batching(fip, synthetic, torch, dev, local))
        forms.update(run_batching_reference_shape(fip, torch, d, snap, dev, local, value))

    # ---- serving form: 4 beams, Poisson arrivals, HBM budget (rank 0) ----
    if rank == 0 and not args.no_forms:
        from fastimagingpipe_b200 import serving
        beams = [synthetic.config_reference(n_ant=256, image_size=1024, cell_size=2.9089e-5,
                                            n_snap=6, seed=11),
                 synthetic.config_reference(image_size=2048, cell_size=1.4544e-5, n_snap=6,
                                            seed=12),
                 synthetic.config_reference(n_snap=6, seed=13),
                 synthetic.config_reference(n_snap=6, seed=14)]
        rates = [200.0, 100.0, 50.0, 20.0]
        with fip.Server(150 << 30, slots=4, device=local) as sv:
            ids = [sv.add_beam(s.image_size, s.num_baselines, s.cell_size, s.unit_size)
                   for s in beams]
            serving.run_poisson(sv, ids, beams, rates, 0.3, seed=1)  # warm-up
            sres = serving.run_poisson(sv, ids, beams, rates, 3.0, seed=2)
            sres["hbm_reserved_gb"] = sv.reserved_bytes / 2**30
            # Saturation sweep: the same mix at growing offered load, past
            # what the GPU can serve (throughput flattens, latency grows).
            sweep = []
            for factor in (1, 4, 16, 32, 64):
                st0 = sv.stats()
                r = serving.run_poisson(sv, ids, beams, [x * factor for x in rates], 1.5,
                                        seed=10 + factor)
                st1 = sv.stats()
                steps = st1["steps"] - st0["steps"]
                sweep.append({"offered_per_s": sum(rates) * factor,
                              "throughput": r["throughput"], "p50_ms": r["p50_ms"],
                              "p99_ms": r["p99_ms"], "refused": r["refused"],
                              "snapshots_per_launch": (st1["snapshots"] - st0["snapshots"]) /
                                                      steps if steps else None})
            sres["saturation_sweep"] = sweep
        sres["config"] = ("beams 1024^2/32,640 bl, 2048^2/130,816, 4096^2/130,816 x2; Poisson "
                          "200/100/50/20 snapshots/s (x1..x64 in the sweep, 1.5 s each); HBM "
                          "budget 150 GB; 4 slots; merged launches of up to 8 snapshots")
        forms["serving"] = sres

    # ---- CPU baseline and FP64 errors (rank 0, N = 1) ----
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, ref64 = cpu_baseline(snap)
        line["cpu_baseline"] = cb
        plain = result.cpu().numpy().reshape(u, u)
        line["tlisi_error_vs_fp64"] = {"plain": float(np.abs(plain - ref64).max())}
        for name in ("precise_f16", "precise_f32"):
            if name in forms:
                line["tlisi_error_vs_fp64"][name] = float(
                    np.abs(forms[name]["tlisi"] - ref64).max())
        line["tlisi_error_vs_fp64"]["max_1_minus_tlisi_fp64"] = float((1 - ref64).max())
        # The same shape with the transient in the third snapshot, where it
        # survives D = ||I1 - I2| - |I2 - I3|| (1 - tLISI = 0.27 at its tile):
        # errors measured on a matrix whose range can tell right from wrong.
        import oracle
        third = synthetic.config_reference(seed=1, transient_snapshot=2)
        t64, _, _ = oracle.fipipe(third, "f64")
        disc = {"max_1_minus_tlisi_fp64": float((1 - t64).max())}
        for name, kw in (("plain", {}),
                         ("precise_f16", dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16))):
            with fip.Imager(n, nb, cell, t, device=local, **kw) as im3:
                got = im3.pipe_host(third.vis_re, third.vis_im, third.B, third.V, nb)
            disc[name] = float(np.abs(got - t64).max())
        line["tlisi_error_vs_fp64_transient_third"] = disc
    if line is not None:
        for f in forms.values():
            f.pop("tlisi", None)
        if forms:
            line["forms"] = forms
        print(json.dumps(line), flush=True)
    im.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
