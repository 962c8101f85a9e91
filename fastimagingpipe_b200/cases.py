"""Representative small cases of the imaging path, for profiling and smoke runs.

    python -m fastimagingpipe_b200.cases batch-mfs [plain|precise]
        four 8-channel (130-150 MHz) snapshots of 4096^2 from 512 antennas,
        0-30 % flagged (the batching configuration's 4096^2 half), imaged by one
        Batch call twice (the second call is the steady state); about 2 GB of
        device memory.
    python -m fastimagingpipe_b200.cases trigger-window [plain|precise]
        the sliding-window trigger over 18 seeded 4096^2 images (16 triples,
        tile 32), streamed and per-triple (fip_set_trigger_streaming).

    python -m fastimagingpipe_b200.cases fipipe [plain|precise]
        three device-resident three-snapshot calls (fip_pipe_device) at
        4096^2, 130,816 baselines, tile 32 (precise: FP16 storage).

Each prints one line and exits 0; inputs are seeded synthetic data.
"""
import sys


def batch_mfs(form: str) -> str:
    import torch
    import fastimagingpipe_b200 as fip
    from fastimagingpipe_b200 import synthetic
    dev = torch.device("cuda:0")
    snaps = synthetic.config_batching(4096, n_snap=2, n_chan=8, seed=20 + 4096)
    d = [{k: torch.tensor(getattr(x, k), device=dev) for k in ("vis_re", "vis_im", "B", "V")}
         for x in snaps]
    idx = [0, 1, 0, 1]
    args = ([d[i]["vis_re"] for i in idx], [d[i]["vis_im"] for i in idx],
            [d[i]["B"] for i in idx], [d[i]["V"] for i in idx], [snaps[i].nb for i in idx])
    kw = {} if form == "plain" else dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)
    with fip.Batch(4096, max(s.nb for s in snaps), snaps[0].cell_size, 32, 4, **kw) as b:
        res = torch.zeros((4, 128 * 128), device=dev)
        for _ in range(2):
            b.reset()
            b.image(*args, res)
        torch.cuda.synchronize()
        b.check()
    return f"batch-mfs {form}: 4 snapshots, nb {[snaps[i].nb for i in idx]}"


def trigger_window(form: str) -> str:
    import torch
    import fastimagingpipe_b200 as fip
    dev = torch.device("cuda:0")
    n, t, count = 4096, 32, 18
    g = torch.Generator(device=dev).manual_seed(7)
    x = torch.rand(count, n, n, device=dev, generator=g)
    mx = x.reshape(count, -1).max(dim=1).values.contiguous()
    out = torch.zeros((count - 2) * (n // t) ** 2, device=dev)
    f = fip.FORM_PLAIN if form == "plain" else fip.FORM_PRECISE
    prev = fip.set_trigger_streaming(True)
    try:
        with fip.Imager(n, 16, 1e-5, t, form=f) as im:
            for stream in (True, False):
                fip.set_trigger_streaming(stream)
                im.trigger_window(x, mx, count, out)
            torch.cuda.synchronize()
    finally:
        fip.set_trigger_streaming(prev)
    return f"trigger-window {form}: {count - 2} triples, min tLISI {float(out.min()):.4f}"


def fipipe(form: str) -> str:
    import torch
    import fastimagingpipe_b200 as fip
    from fastimagingpipe_b200 import synthetic
    dev = torch.device("cuda:0")
    snap = synthetic.config_reference(transient_snapshot=2)
    n, nb, t = snap.image_size, snap.num_baselines, snap.unit_size
    d = {k: torch.tensor(getattr(snap, k), device=dev) for k in ("vis_re", "vis_im", "B", "V")}
    out = torch.zeros((n // t) ** 2, device=dev)
    kw = {} if form == "plain" else dict(form=fip.FORM_PRECISE, vis_storage=fip.STORE_F16)
    with fip.Imager(n, nb, snap.cell_size, t, **kw) as im:
        for _ in range(3):
            im.pipe_device(d["vis_re"], d["vis_im"], d["B"], d["V"], nb, out)
        torch.cuda.synchronize()
        im.check()
    return f"fipipe {form}: min tLISI {float(out.min()):.4f}"


CASES = {"batch-mfs": batch_mfs, "trigger-window": trigger_window, "fipipe": fipipe}


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] not in CASES:
        print(__doc__)
        return 2
    form = argv[1] if len(argv) > 1 else "plain"
    if form not in ("plain", "precise"):
        print("form: plain or precise")
        return 2
    print(CASES[argv[0]](form))
    return 0


if __name__ == "__main__":
    sys.exit(main())
