"""ctypes front end of the CPU oracle (oracle/fip_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py for the CPU-baseline leg.  The product package never
imports it.

Every function takes/returns numpy arrays.  `prec` selects the FP64 oracle
("f64", the accuracy target) or the FP32 restatement in the reference's
operation order ("f32").
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_sz = ctypes.c_size_t


def build() -> str:
    """Compile liboracle.so with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        for p, rp in (("f64", _f64p), ("f32", _f32p)):
            getattr(L, f"oracle_grid_size_{p}").restype = _sz
            getattr(L, f"oracle_grid_size_{p}").argtypes = [_sz]
            getattr(L, f"oracle_taper_{p}").argtypes = [rp, _sz, _sz]
            getattr(L, f"oracle_fft1d_{p}").argtypes = [rp, rp, _sz, ctypes.c_int]
            getattr(L, f"oracle_grid_{p}").argtypes = [rp, _f32p, _f32p, _f32p, _f32p, _sz, _sz,
                                                       ctypes.c_float]
            getattr(L, f"oracle_pixel_targets_{p}").argtypes = [rp, _f32p, _sz, ctypes.c_float]
            f = getattr(L, f"oracle_image_snapshot_{p}")
            f.restype = ctypes.c_double if p == "f64" else ctypes.c_float
            f.argtypes = [rp, ctypes.c_void_p, _f32p, _f32p, _f32p, _f32p, _sz, _sz,
                          ctypes.c_float]
            getattr(L, f"oracle_tlisi_{p}").argtypes = [rp, rp, rp, rp, rp, _sz, _sz]
            getattr(L, f"oracle_fipipe_{p}").argtypes = [rp, ctypes.c_void_p, ctypes.c_void_p,
                                                         _f32p, _f32p, _f32p, _f32p, _sz, _sz,
                                                         ctypes.c_float, _sz]
            getattr(L, f"oracle_plane_fit_{p}").argtypes = [_f64p, _f64p, _f32p, _f32p, _sz, _sz]
            getattr(L, f"oracle_collapse_{p}").argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p,
                                                           _f32p, _u8p, _u8p, _f32p, _f32p, _sz]
            getattr(L, f"oracle_num_threads_{p}").restype = ctypes.c_int
        _LIB = L
    return _LIB


def _dt(prec):
    return np.float64 if prec == "f64" else np.float32


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def grid_size(image_size: int) -> int:
    return int(lib().oracle_grid_size_f64(image_size))


def num_threads() -> int:
    return int(lib().oracle_num_threads_f64())


def taper(image_size: int, prec: str = "f64") -> np.ndarray:
    g = grid_size(image_size)
    out = np.zeros(image_size // 2 + 1, _dt(prec))
    getattr(lib(), f"oracle_taper_{prec}")(out, image_size, g)
    return out


def fft1d(x: np.ndarray, sign: int = +1, prec: str = "f64") -> np.ndarray:
    x = np.asarray(x, np.complex128 if prec == "f64" else np.complex64)
    inp = np.ascontiguousarray(x.view(_dt(prec)))
    out = np.zeros_like(inp)
    getattr(lib(), f"oracle_fft1d_{prec}")(inp, out, x.shape[0], sign)
    return out.view(np.complex128 if prec == "f64" else np.complex64)


def grid(B, vr, vi, V, nb, image_size, cell, prec="f64") -> np.ndarray:
    g = grid_size(image_size)
    out = np.zeros(g * g * 2, _dt(prec))
    getattr(lib(), f"oracle_grid_{prec}")(out, _f32(B), _f32(vr), _f32(vi), _f32(V), nb, g, cell)
    return out.view(np.complex128 if prec == "f64" else np.complex64).reshape(g, g)


def pixel_targets(V, image_size, cell, prec="f64") -> np.ndarray:
    out = np.zeros(image_size * image_size * 2, _dt(prec))
    getattr(lib(), f"oracle_pixel_targets_{prec}")(out, _f32(V), image_size, cell)
    return out.reshape(image_size, image_size, 2)


def image_snapshot(B, vr, vi, V, nb, image_size, cell, prec="f64", want_pre=False):
    """-> (dirty [N,N], max, dirty_pre [N,N] or None)."""
    n = image_size
    dirty = np.zeros(n * n, _dt(prec))
    pre = np.zeros(n * n, _dt(prec)) if want_pre else None
    mx = getattr(lib(), f"oracle_image_snapshot_{prec}")(
        dirty, pre.ctypes.data if pre is not None else None, _f32(B), _f32(vr), _f32(vi),
        _f32(V), nb, n, cell)
    return dirty.reshape(n, n), float(mx), (pre.reshape(n, n) if pre is not None else None)


def tlisi(I1, I2, I3, maxall, unit_size, prec="f64") -> np.ndarray:
    n = I1.shape[0]
    u = n // unit_size
    out = np.zeros(u * u, _dt(prec))
    c = lambda a: np.ascontiguousarray(a, _dt(prec))
    getattr(lib(), f"oracle_tlisi_{prec}")(out, c(I1), c(I2), c(I3), c(maxall), n, unit_size)
    return out.reshape(u, u)


def fipipe(snap, prec="f64", want_images=False):
    """The reference FIpipe computation on a synthetic.SnapshotSet.
    -> (tlisi [U,U], images [3,N,N] or None, maxall [3])."""
    n, t = snap.image_size, snap.unit_size
    u = n // t
    res = np.zeros(u * u, _dt(prec))
    imgs = np.zeros(3 * n * n, _dt(prec)) if want_images else None
    mx = np.zeros(3, _dt(prec))
    getattr(lib(), f"oracle_fipipe_{prec}")(
        res, imgs.ctypes.data if imgs is not None else None, mx.ctypes.data, _f32(snap.vis_re),
        _f32(snap.vis_im), _f32(snap.B), _f32(snap.V), snap.num_baselines, n, snap.cell_size, t)
    return res.reshape(u, u), (imgs.reshape(3, n, n) if imgs is not None else None), mx


def locate(tlisi, image_size, unit_size, cell, threshold):
    """Transient locations of a tLISI matrix (the rule fip_locate_transients
    states; the reference names its output locations.fits, README.md:41, and
    leaves the reduction to the user): tiles below `threshold` that are the
    strict minimum of their 3 x 3 neighbourhood (ties to the lower index),
    refined to the neighbourhood's centroid of max(0, 1 - tLISI), sorted
    deepest first.  Plain Python loops over the tiles (small matrices)."""
    t = np.asarray(tlisi, np.float32)
    u = t.shape[0]
    out = []
    h1 = image_size // 2 + 1
    for r in range(u):
        for c in range(u):
            v = t[r, c]
            if not v < threshold:
                continue
            ws = wr = wc = 0.0
            ok = True
            for dr in (-1, 0, 1):
                for dc in (-1, 0, 1):
                    rr, cc = r + dr, c + dc
                    if not (0 <= rr < u and 0 <= cc < u):
                        continue
                    w = t[rr, cc]
                    if (rr, cc) != (r, c) and (w < v or (w == v and rr * u + cc < r * u + c)):
                        ok = False
                    d = max(0.0, 1.0 - float(w)) if w == w else 0.0
                    ws += d
                    wr += d * dr
                    wc += d * dc
            if not ok:
                continue
            fr = r + (wr / ws if ws > 0 else 0.0)
            fc = c + (wc / ws if ws > 0 else 0.0)
            row = fr * unit_size + 0.5 * (unit_size - 1)
            col = fc * unit_size + 0.5 * (unit_size - 1)
            out.append((r, c, float(v), row, col, -cell * (col - h1), cell * (row - h1)))
    out.sort(key=lambda e: (e[2], e[0] * u + e[1]))
    return out


def plane_fit(uvw_m, freqs_hz):
    """uvw [rows,3] metres, freqs [chans] Hz -> (B [rows*chans,2], V [3,3]) FP64."""
    uvw = _f32(uvw_m).reshape(-1, 3)
    fr = _f32(np.atleast_1d(freqs_hz))
    rows, chans = uvw.shape[0], fr.shape[0]
    B = np.zeros(rows * chans * 2, np.float64)
    V = np.zeros(9, np.float64)
    lib().oracle_plane_fit_f64(B, V, uvw, fr, rows, chans)
    return B.reshape(-1, 2), V.reshape(3, 3)


def collapse(v0r, v0i, v3r, v3i, f0, f3, w0, w3):
    ns = len(v0r)
    o_re = np.zeros(ns, np.float32)
    o_im = np.zeros(ns, np.float32)
    u8 = lambda a: np.ascontiguousarray(a, np.uint8)
    lib().oracle_collapse_f64(o_re, o_im, _f32(v0r), _f32(v0i), _f32(v3r), _f32(v3i), u8(f0),
                              u8(f3), _f32(w0), _f32(w3), ns)
    return o_re, o_im
