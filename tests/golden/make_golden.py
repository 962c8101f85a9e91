"""Generates the golden fixtures of the reference's own implementation.

Runs the reference's FIPkernels.cu, recompiled for sm_100a by
`make -C oracle ref` (oracle/_ref/libfipref.so), on seeded synthetic inputs
and stores its outputs here:

    python tests/golden/make_golden.py      # needs a GPU and oracle/_ref

The inputs are regenerated from their seeds by fastimagingpipe_b200.synthetic;
a SHA-256 of the input bytes is stored to detect drift.  Outputs:
  reference_tiny.npz   128^2, tile 16: full images, maxima, tLISI, the
                       pixel targets and pre-reprojection image of snapshot 0
  reference_small.npz  512^2, tile 16: tLISI, maxima, row/column sums and a
                       64x64 crop around each image maximum, pixel targets at
                       4096 seeded pixels
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from fastimagingpipe_b200 import synthetic  # noqa: E402
from oracle import reference as ref  # noqa: E402


def input_digest(snap):
    h = hashlib.sha256()
    for a in (snap.vis_re, snap.vis_im, snap.B, snap.V):
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    return h.hexdigest()


def images(snap):
    out, mx, pre0 = [], [], None
    for k in range(3):
        vr, vi, B, V = snap.snapshot(k)
        d, pre, m = ref.image_snapshot(vr, vi, B, V, snap.num_baselines, snap.image_size,
                                       snap.cell_size)
        out.append(d)
        mx.append(m)
        if k == 0:
            pre0 = pre
    return np.stack(out), np.array(mx, np.float32), pre0


def main():
    assert ref.available(), "build oracle/_ref first: make -C oracle ref"
    tiny = synthetic.config_tiny(transient_snapshot=2)
    imgs, mx, pre0 = images(tiny)
    np.savez_compressed(os.path.join(HERE, "reference_tiny.npz"),
                        digest=input_digest(tiny), images=imgs, maxall=mx,
                        tlisi=ref.fipipe(tiny), tlisi_from_images=ref.trigger(*imgs, mx, tiny.unit_size),
                        targets0=ref.pixel_targets(tiny.V[:9], tiny.image_size, tiny.cell_size),
                        pre0=pre0)
    small = synthetic.config_small(transient_snapshot=2)
    imgs, mx, _ = images(small)
    n = small.image_size
    crops, origins = [], []
    for k in range(3):
        r, c = np.unravel_index(np.argmax(imgs[k]), imgs[k].shape)
        r0 = int(min(max(r - 32, 0), n - 64))
        c0 = int(min(max(c - 32, 0), n - 64))
        crops.append(imgs[k][r0:r0 + 64, c0:c0 + 64])
        origins.append((r0, c0))
    rng = np.random.default_rng(11)
    pix = rng.integers(0, n, size=(4096, 2))
    tg = ref.pixel_targets(small.V[:9], n, small.cell_size)
    np.savez_compressed(os.path.join(HERE, "reference_small.npz"),
                        digest=input_digest(small), tlisi=ref.fipipe(small), maxall=mx,
                        row_sums=imgs.sum(axis=2), col_sums=imgs.sum(axis=1),
                        crops=np.stack(crops), crop_origins=np.array(origins),
                        target_pixels=pix, targets=tg[pix[:, 0], pix[:, 1]])
    print("golden fixtures written")


if __name__ == "__main__":
    main()
