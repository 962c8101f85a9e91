"""ctypes front end of the reference's own CUDA build (oracle/_ref/libfipref.so,
and its GPU preprocessing in oracle/_ref/libfippre.so).

TEST INFRASTRUCTURE ONLY: the reference's FIPkernels.cu and
SVDPreprocessKernels.cu recompiled for sm_100a by `make -C oracle ref` (the
sources are read where they lie at build time; the built libraries travel with
the repository).  Used by the GPU parity tests and by bench.py's reference
arm; never by the product.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libfipref.so")
PRE_LIB_PATH = os.path.join(_HERE, "_ref", "libfippre.so")
_LIB = None
_PRE = None


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


def preprocess_available() -> bool:
    return os.path.exists(PRE_LIB_PATH)


def preprocess(uvw_m, freqs_hz, v0, v3, flag0, flag3, weight0, weight3):
    """The reference's GPU preprocessing (SVDPreprocessKernels.cu:255-500):
    uvw [rows][3] metres, freqs [chans] Hz, complex polarisations 0 and 3,
    uint8 flags and weights [rows * chans] (sample row + chan * rows).
    Returns B [samples][2], V [3][3], and the collapsed visibilities
    (real, imaginary)."""
    global _PRE
    if _PRE is None:
        L = ctypes.CDLL(PRE_LIB_PATH)
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.ref_preprocess.argtypes = [sz, sz] + [vp] * 14
        L.ref_preprocess.restype = ctypes.c_int
        _PRE = L
    uvw = _f(uvw_m).reshape(-1, 3)
    freqs = _f(freqs_hz)
    rows, chans = uvw.shape[0], freqs.shape[0]
    ns = rows * chans
    arrs = [_f(np.real(v0)), _f(np.imag(v0)), _f(np.real(v3)), _f(np.imag(v3))]
    flags = [np.ascontiguousarray(f, dtype=np.uint8) for f in (flag0, flag3)]
    weights = [_f(w) for w in (weight0, weight3)]
    B = np.zeros((ns, 2), np.float32)
    V = np.zeros(9, np.float32)
    vr = np.zeros(ns, np.float32)
    vi = np.zeros(ns, np.float32)
    rc = _PRE.ref_preprocess(rows, chans, uvw.ctypes.data, freqs.ctypes.data,
                             *(a.ctypes.data for a in arrs), *(f.ctypes.data for f in flags),
                             *(w.ctypes.data for w in weights), B.ctypes.data, V.ctypes.data,
                             vr.ctypes.data, vi.ctypes.data)
    if rc != 0:
        raise RuntimeError("the reference's preprocessing failed")
    return B, V.reshape(3, 3), vr, vi
