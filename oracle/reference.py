"""ctypes front end of the reference's own CUDA build (oracle/_ref/libfipref.so).

TEST INFRASTRUCTURE ONLY: the reference's FIPkernels.cu recompiled for sm_100a
by `make -C oracle ref` (the sources are read where they lie at build time; the
built library travels with the repository).  Used by the GPU parity tests and
by bench.py's reference arm; never by the product.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libfipref.so")
_LIB = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, fp = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float
        L.ref_fipipe.argtypes = [vp, vp, vp, vp, vp, sz, sz, sz, fp, sz]
        L.ref_image_snapshot.argtypes = [vp, vp, vp, vp, sz, sz, fp, vp, vp, vp]
        L.ref_trigger.argtypes = [vp, vp, vp, vp, sz, sz, vp]
        L.ref_pixel_targets.argtypes = [vp, sz, fp, vp]
        _LIB = L
    return _LIB


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def fipipe(snap) -> np.ndarray:
    """The unmodified reference FIpipe on a synthetic.SnapshotSet."""
    n, t = snap.image_size, snap.unit_size
    u = n // t
    out = np.zeros((u, u), np.float32)
    arrs = [_f(snap.vis_re), _f(snap.vis_im), _f(snap.B), _f(snap.V)]
    lib().ref_fipipe(*(a.ctypes.data for a in arrs), out.ctypes.data, snap.num_baselines, n,
                     snap.num_snapshots, snap.cell_size, t)
    return out


def image_snapshot(vr, vi, B, V, nb, n, cell):
    """Reference kernels of one snapshot -> (dirty [N,N], dirty_pre [N,N], max)."""
    dirty = np.zeros((n, n), np.float32)
    pre = np.zeros((n, n), np.float32)
    mx = np.zeros(1, np.float32)
    arrs = [_f(vr), _f(vi), _f(B), _f(V)]
    st = lib().ref_image_snapshot(*(a.ctypes.data for a in arrs), nb, n, cell, dirty.ctypes.data,
                                  pre.ctypes.data, mx.ctypes.data)
    if st != 0:
        raise RuntimeError(f"ref_image_snapshot failed ({st})")
    return dirty, pre, float(mx[0])


def trigger(I1, I2, I3, max3, t) -> np.ndarray:
    n = I1.shape[0]
    u = n // t
    out = np.zeros((u, u), np.float32)
    arrs = [_f(I1), _f(I2), _f(I3), _f(max3)]
    st = lib().ref_trigger(*(a.ctypes.data for a in arrs), n, t, out.ctypes.data)
    if st != 0:
        raise RuntimeError(f"ref_trigger failed ({st})")
    return out


def pixel_targets(V, n, cell) -> np.ndarray:
    """coordschange + p2p output, re-indexed to [row j][column i][2] and
    centred (LL, MM) like the oracle's pixel_targets."""
    oi = np.zeros(n * n * 2, np.float32)
    st = lib().ref_pixel_targets(_f(V).ctypes.data, n, cell, oi.ctypes.data)
    if st != 0:
        raise RuntimeError(f"ref_pixel_targets failed ({st})")
    oi = oi.reshape(n, n, 2)  # [i][j][2] (FIPkernels.cu:296)
    return np.ascontiguousarray(oi.transpose(1, 0, 2)) - np.float32(n // 2)
