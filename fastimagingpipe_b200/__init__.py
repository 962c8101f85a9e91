"""B200-native snapshot imaging + tLISI trigger (FastImagingPipe's hot path).

Python mirror of the reference's entry point over the C ABI of
libfip_b200.so (include/fip.h):

* ``FIpipe(vis_re, vis_im, B, V, num_baselines, image_size, num_snapshots,
  cell_size, unit_size)`` -> tLISI matrix, the same arguments and meaning as
  the reference's ``FIpipe`` (FIPkernels.cu:554-557; pipe_interface.cpp:181),
  host arrays in, host array out;
* ``Imager``: persistent device state for one image size, device-pointer
  calls for snapshot imaging, the trigger, sequences and the FIpipe shape;
* ``plane_project`` / ``collapse_visibilities``: the on-device preprocessing
  (SVDPreprocessKernels.cu).

The CUDA library is required: nothing here falls back to the CPU.  Device
buffers may be passed as integer addresses or as objects exposing
``data_ptr()`` (torch tensors).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfip_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "sharedlibrary_gpu")

FORM_PLAIN = 0
FORM_PRECISE = 1
STORE_F32, STORE_F16, STORE_BF16 = 0, 1, 2
REPROJECT_GATHER, REPROJECT_SCATTER = 0, 1

_lib = None


class FipError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"fip status {status}: {message}")
        self.status = status


class ImagerConfig(ctypes.Structure):
    _fields_ = [("image_size", ctypes.c_size_t), ("max_baselines", ctypes.c_size_t),
                ("unit_size", ctypes.c_size_t), ("cell_size", ctypes.c_float),
                ("form", ctypes.c_int), ("vis_storage", ctypes.c_int),
                ("device", ctypes.c_int), ("reproject", ctypes.c_int)]


class Location(ctypes.Structure):
    """fip_location: one transient location (see locate_transients)."""
    _fields_ = [("tile_row", ctypes.c_int32), ("tile_col", ctypes.c_int32),
                ("tlisi", ctypes.c_float), ("row", ctypes.c_float), ("col", ctypes.c_float),
                ("x", ctypes.c_float), ("y", ctypes.c_float)]


LOCATION_DTYPE = np.dtype([("tile_row", "<i4"), ("tile_col", "<i4"), ("tlisi", "<f4"),
                           ("row", "<f4"), ("col", "<f4"), ("x", "<f4"), ("y", "<f4")])


class RawVis(ctypes.Structure):
    """fip_raw_vis: device pointers of one snapshot's raw polarisations 0 and 3,
    their flags (uint8, nonzero = flagged) and weights."""
    _fields_ = [(k, ctypes.c_void_p) for k in ("v0_re", "v0_im", "v3_re", "v3_im", "flag0",
                                              "flag3", "weight0", "weight3")]


def lib() -> ctypes.CDLL:
    """Loads libfip_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`python -m fastimagingpipe_b200.build` (there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, fp = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float
        L.fip_last_error.restype = ctypes.c_char_p
        L.fip_status_string.restype = ctypes.c_char_p
        L.fip_status_string.argtypes = [ctypes.c_int]
        L.fip_version.restype = ctypes.c_char_p
        L.fip_pipe.argtypes = [vp, vp, vp, vp, vp, sz, sz, sz, fp, sz]
        L.fip_imager_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ImagerConfig)]
        L.fip_imager_destroy.argtypes = [vp]
        L.fip_imager_device_bytes.argtypes = [vp]
        L.fip_imager_device_bytes.restype = sz
        L.fip_image_snapshot.argtypes = [vp, vp, vp, vp, vp, sz, vp, vp, vp]
        L.fip_trigger.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.fip_pipe_device.argtypes = [vp, vp, vp, vp, vp, sz, vp, vp]
        L.fip_imager_image.argtypes = [vp, ctypes.c_int]
        L.fip_imager_image.restype = vp
        L.fip_imager_check.argtypes = [vp, vp]
        L.fip_server_set_max_step.argtypes = [vp, ctypes.c_int]
        L.fip_server_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_long),
                                       ctypes.POINTER(ctypes.c_long)]
        L.fip_batch_image_slots.argtypes = [vp, vp, vp, vp, vp, vp, sz, vp, vp]
        L.fip_batch_set_profiling.argtypes = [vp, ctypes.c_int]
        L.fip_batch_phase_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_long)]
        L.fip_locate_transients.argtypes = [vp, sz, sz, fp, fp, vp, sz,
                                             ctypes.POINTER(sz), vp]
        L.fip_image_snapshot_raw.argtypes = [vp, ctypes.POINTER(RawVis), vp, vp, sz, vp, vp, vp]
        L.fip_batch_check.argtypes = [vp, vp]
        L.fip_batch_create_sequences.argtypes = [ctypes.POINTER(vp), vp, sz, sz]
        L.fip_batch_image_sequences.argtypes = [vp, vp, vp, vp, vp, vp, vp, sz, vp, vp, vp]
        L.fip_batch_autotune_sequences.argtypes = [vp, vp, vp, vp, vp, vp, vp, sz, vp]
        L.fip_batch_sequence_tuning.argtypes = [vp, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 4
        L.fip_set_trigger_streaming.argtypes = [ctypes.c_int]
        L.fip_trigger_window.argtypes = [vp, vp, vp, sz, vp, vp]
        L.fip_pipe_host.argtypes = [vp, vp, vp, vp, vp, sz, sz, vp]
        L.fip_pixel_targets.argtypes = [vp, vp, vp, ctypes.c_int, vp]
        L.fip_plane_project.argtypes = [vp, vp, sz, sz, vp, vp, vp]
        L.fip_collapse_visibilities.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]
        L.fip_image_sequence.argtypes = [vp, vp, vp, vp, vp, vp, sz, sz, vp, vp]
        L.fip_imager_set_profiling.argtypes = [vp, ctypes.c_int]
        L.fip_imager_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_long), ctypes.c_int]
        L.fip_stage_name.argtypes = [ctypes.c_int]
        L.fip_stage_name.restype = ctypes.c_char_p
        L.fip_stage_count.restype = ctypes.c_int
        L.fip_imager_kernel_launches.argtypes = [vp]
        L.fip_imager_kernel_launches.restype = ctypes.c_ulonglong
        L.fip_imager_band.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_uint)]
        L.fip_imager_grid_side.argtypes = [vp]
        L.fip_imager_autotune.argtypes = [vp, vp, vp, vp, vp, sz, vp]
        L.fip_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ImagerConfig), sz]
        L.fip_batch_destroy.argtypes = [vp]
        L.fip_batch_device_bytes.argtypes = [vp]
        L.fip_batch_device_bytes.restype = sz
        L.fip_batch_kernel_launches.argtypes = [vp]
        L.fip_batch_kernel_launches.restype = ctypes.c_ulonglong
        L.fip_batch_reset.argtypes = [vp]
        L.fip_batch_image.argtypes = [vp, vp, vp, vp, vp, vp, sz, vp, ctypes.POINTER(sz), vp]
        L.fip_batch_autotune.argtypes = [vp, vp, vp, vp, vp, vp, sz, vp]
        L.fip_batch_tuning.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 4
        L.fip_imager_tuning.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 4
        L.fip_imager_set_tuning.argtypes = [vp] + [ctypes.c_int] * 4
        L.fip_grid_snapshot.argtypes = [vp, vp, vp, vp, vp, sz, vp, vp]
        L.fip_grid_snapshot_noalloc.argtypes = [vp, vp, vp, vp, sz, sz, fp, vp, vp]
        L.fip_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, sz, ctypes.c_int, sz]
        L.fip_server_destroy.argtypes = [vp]
        L.fip_server_add_beam.argtypes = [vp, ctypes.POINTER(ImagerConfig),
                                          ctypes.POINTER(ctypes.c_int)]
        L.fip_server_reserved_bytes.argtypes = [vp]
        L.fip_server_reserved_bytes.restype = sz
        L.fip_server_submit.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, sz,
                                        ctypes.POINTER(ctypes.c_long)]
        L.fip_server_wait.argtypes = [vp, ctypes.c_long, ctypes.c_double,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_long),
                                      ctypes.POINTER(ctypes.c_int), vp, sz,
                                      ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def _check(status: int):
    if status != 0:
        raise FipError(status, lib().fip_last_error().decode(errors="replace"))


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    raise TypeError(f"expected a device address or a tensor, got {type(x)!r}")


def _stream(s) -> int:
    if s is None:
        return 0
    if isinstance(s, int):
        return s
    return int(getattr(s, "cuda_stream", s))


def version() -> str:
    return lib().fip_version().decode()


def FIpipe(Visreal, Visimag, Bin, Vin, num_baselines: int, image_size: int,
           num_snapshots: int, cell_size: float, unit_size: int) -> np.ndarray:
    """The reference's FIpipe (FIPkernels.cu:554) on host arrays: images the
    first three snapshots and returns the (N/T, N/T) tLISI matrix."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (Visreal, Visimag, Bin, Vin)]
    nb, n, s, t = int(num_baselines), int(image_size), int(num_snapshots), int(unit_size)
    if arrs[0].size < s * nb or arrs[1].size < s * nb or arrs[2].size < s * nb * 2 or \
            arrs[3].size < s * 9:
        raise ValueError("input arrays are smaller than num_snapshots x num_baselines")
    u = n // t if t > 0 else 0
    out = np.zeros((u, u), np.float32)
    _check(lib().fip_pipe(*(a.ctypes.data for a in arrs), out.ctypes.data, nb, n, s,
                          float(cell_size), t))
    return out


class Imager:
    """Persistent imager (fip_imager) for one image size."""

    def __init__(self, image_size: int, max_baselines: int, cell_size: float,
                 unit_size: int = 0, form: int = FORM_PLAIN, vis_storage: int = STORE_F32,
                 device: int = 0, reproject: int = REPROJECT_GATHER):
        self.cfg = ImagerConfig(image_size, max_baselines, unit_size, cell_size, form,
                                vis_storage, device, reproject)
        h = ctypes.c_void_p()
        _check(lib().fip_imager_create(ctypes.byref(h), ctypes.byref(self.cfg)))
        self._h = h
        self.image_size = image_size
        self.unit_size = unit_size
        self.max_baselines = max_baselines

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().fip_imager_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def device_bytes(self) -> int:
        return int(lib().fip_imager_device_bytes(self._h))

    def set_profiling(self, enable: bool = True):
        """Per-stage device timing with CUDA events (resets the totals)."""
        _check(lib().fip_imager_set_profiling(self._h, int(enable)))

    def stage_times(self) -> dict:
        """{stage: (total_ms, launches)} accumulated since set_profiling(True)."""
        n = int(lib().fip_stage_count())
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_long * n)()
        _check(lib().fip_imager_stage_times(self._h, ms, cnt, n))
        return {lib().fip_stage_name(k).decode(): (ms[k], cnt[k]) for k in range(n)}

    @property
    def kernel_launches(self) -> int:
        return int(lib().fip_imager_kernel_launches(self._h))

    @property
    def grid_side(self) -> int:
        return int(lib().fip_imager_grid_side(self._h))

    def autotune(self, vis_re, vis_im, B, V, nb: int, stream=None) -> dict:
        """Times the transform's values per thread and the gridder's CTAs per SM on
        this snapshot (device buffers) and keeps the fastest; returns the choice.
        Overwrites the trigger ring: call it before a run of snapshots."""
        _check(lib().fip_imager_autotune(self._h, _ptr(vis_re), _ptr(vis_im), _ptr(B), _ptr(V),
                                         nb, _stream(stream)))
        return self.tuning()

    def set_tuning(self, fft_values_per_thread: int = 0, fft_split: int = 0,
                   grid_ctas_per_sm: int = 0, fft_direct: int = 0):
        _check(lib().fip_imager_set_tuning(self._h, fft_values_per_thread, fft_split,
                                           fft_direct, grid_ctas_per_sm))

    def tuning(self) -> dict:
        e, sp, dr, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().fip_imager_tuning(self._h, ctypes.byref(e), ctypes.byref(sp),
                                       ctypes.byref(dr), ctypes.byref(c)))
        return {"fft_values_per_thread": int(e.value), "fft_split": int(sp.value),
                "fft_direct": int(dr.value), "grid_ctas_per_sm": int(c.value)}

    def band(self):
        """(max |r1|, max half-plane column) of the last gridded snapshot."""
        a, b = ctypes.c_uint(), ctypes.c_uint()
        _check(lib().fip_imager_band(self._h, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def image_snapshot(self, vis_re, vis_im, B, V, nb: int, image, image_max=None, stream=None):
        _check(lib().fip_image_snapshot(self._h, _ptr(vis_re), _ptr(vis_im), _ptr(B), _ptr(V), nb,
                                        _ptr(image), _ptr(image_max), _stream(stream)))

    def image_snapshot_raw(self, v0_re, v0_im, v3_re, v3_im, flag0, flag3, weight0, weight3, B,
                           V, nb: int, image, image_max=None, stream=None):
        """image_snapshot from raw polarisations 0 and 3 with flags and weights
        (device arrays of nb samples): the Stokes-I collapse runs inside the
        gridder's load."""
        raw = RawVis(*(_ptr(x) for x in (v0_re, v0_im, v3_re, v3_im, flag0, flag3, weight0,
                                          weight3)))
        _check(lib().fip_image_snapshot_raw(self._h, ctypes.byref(raw), _ptr(B), _ptr(V), nb,
                                            _ptr(image), _ptr(image_max), _stream(stream)))

    def grid_snapshot(self, vis_re, vis_im, B, V, nb: int, grid, stream=None):
        """Gridding stage only: grid [G][G/2+1] complex (2 floats each)."""
        _check(lib().fip_grid_snapshot(self._h, _ptr(vis_re), _ptr(vis_im), _ptr(B), _ptr(V),
                                       nb, _ptr(grid), _stream(stream)))

    def trigger(self, I1, I2, I3, max3, result, stream=None):
        _check(lib().fip_trigger(self._h, _ptr(I1), _ptr(I2), _ptr(I3), _ptr(max3), _ptr(result),
                                 _stream(stream)))

    def trigger_window(self, images, maxima, count: int, results, stream=None):
        """Sliding-window tLISI over `count` consecutive device images ([count][N*N]):
        triple k -> results[k * U*U:(k + 1) * U*U], k < count - 2."""
        _check(lib().fip_trigger_window(self._h, _ptr(images), _ptr(maxima), count, _ptr(results),
                                        _stream(stream)))

    def pipe_device(self, vis_re, vis_im, B, V, nb: int, result, stream=None):
        _check(lib().fip_pipe_device(self._h, _ptr(vis_re), _ptr(vis_im), _ptr(B), _ptr(V), nb,
                                     _ptr(result), _stream(stream)))

    def check(self, stream=None):
        """Raises FipError if a gather reprojection since the last check had a
        tile outside its domain (a folding wide-field geometry)."""
        _check(lib().fip_imager_check(self._h, _stream(stream)))

    def image_ptr(self, k: int) -> int:
        return int(lib().fip_imager_image(self._h, k) or 0)

    def pipe_host(self, vis_re, vis_im, B, V, nb: int, num_snapshots: int = 3) -> np.ndarray:
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vis_re, vis_im, B, V)]
        u = self.image_size // self.unit_size
        out = np.zeros((u, u), np.float32)
        _check(lib().fip_pipe_host(self._h, *(a.ctypes.data for a in arrs), nb, num_snapshots,
                                   out.ctypes.data))
        return out

    def pixel_targets(self, V, out, exact: bool = False, stream=None, evaluated: bool = False):
        """Targets (LL, MM) of every pixel into out [N*N*2]: the plain form's
        FP32 chain as imaged (evaluated=True: step by step, without the
        theta-terms table; the same bits), or the exact closed form."""
        mode = 1 if exact else (2 if evaluated else 0)
        _check(lib().fip_pixel_targets(self._h, _ptr(V), _ptr(out), mode, _stream(stream)))

    def image_sequence(self, vis_re, vis_im, B, V, nb_per_snapshot, nb_stride: int, results,
                       stream=None):
        nbs = np.ascontiguousarray(nb_per_snapshot, dtype=np.uint64)
        _check(lib().fip_image_sequence(self._h, _ptr(vis_re), _ptr(vis_im), _ptr(B), _ptr(V),
                                        nbs.ctypes.data, nb_stride, len(nbs), _ptr(results),
                                        _stream(stream)))


class Batch:
    """Batching form (fip_batch): many snapshots of one image size per
    call, one persistent gridding launch and one batched transform per call,
    replayed as a CUDA graph; the batch carries the sequence's last two images so
    every snapshot with two predecessors yields a tLISI matrix.  Batch.of_sequences
    makes a batch of several sequences of different image sizes, imaged together
    (image_sequences)."""

    def __init__(self, image_size: int, max_baselines: int, cell_size: float, unit_size: int,
                 max_snapshots: int, form: int = FORM_PLAIN, vis_storage: int = STORE_F32,
                 device: int = 0):
        self.cfg = ImagerConfig(image_size, max_baselines, unit_size, cell_size, form,
                                vis_storage, device, REPROJECT_GATHER)
        h = ctypes.c_void_p()
        _check(lib().fip_batch_create(ctypes.byref(h), ctypes.byref(self.cfg), max_snapshots))
        self._h = h
        self.image_size = image_size
        self.unit_size = unit_size
        self.max_snapshots = max_snapshots
        self.sequences = [(image_size, max_baselines, cell_size, unit_size)]

    @classmethod
    def of_sequences(cls, sequences, max_snapshots: int, form: int = FORM_PLAIN,
                     vis_storage: int = STORE_F32, device: int = 0) -> "Batch":
        """A batch of several sequences (fip_batch_create_sequences): `sequences` holds
        (image_size, max_baselines, cell_size, unit_size) per sequence; up to
        max_snapshots of each sequence per call."""
        self = cls.__new__(cls)
        seqs = [tuple(x) for x in sequences]
        cfgs = (ImagerConfig * len(seqs))(*[
            ImagerConfig(n, nb, t, cell, form, vis_storage, device, REPROJECT_GATHER)
            for (n, nb, cell, t) in seqs])
        h = ctypes.c_void_p()
        _check(lib().fip_batch_create_sequences(ctypes.byref(h), ctypes.cast(cfgs, ctypes.c_void_p),
                                                len(seqs), max_snapshots))
        self._h = h
        self.cfg = cfgs[0]
        self.image_size, _, _, self.unit_size = seqs[0]
        self.max_snapshots = max_snapshots
        self.sequences = seqs
        return self

    @staticmethod
    def _arrays(vis_re, vis_im, B, V, nb):
        count = len(nb)
        if not (len(vis_re) == len(vis_im) == len(B) == len(V) == count):
            raise ValueError("one vis_re, vis_im, B, V and nb per snapshot")
        ptrs = lambda xs: (ctypes.c_void_p * count)(*[_ptr(x) for x in xs])
        return (ptrs(vis_re), ptrs(vis_im), ptrs(B), ptrs(V),
                (ctypes.c_size_t * count)(*[int(n) for n in nb]), count)

    def image(self, vis_re, vis_im, B, V, nb, results, stream=None) -> int:
        """Images len(nb) snapshots (per-snapshot device buffers); writes the tLISI
        matrices of the snapshots with two predecessors to `results` (U*U each, in
        order) and returns their number."""
        a = self._arrays(vis_re, vis_im, B, V, nb)
        nr = ctypes.c_size_t()
        _check(lib().fip_batch_image(self._h, *a, _ptr(results), ctypes.byref(nr),
                                     _stream(stream)))
        return int(nr.value)

    def image_sequences(self, sequence, vis_re, vis_im, B, V, nb, results, stream=None) -> list:
        """Images len(nb) snapshots of several sequences in one call: snapshot k
        belongs to sequence sequence[k]; sequence c's tLISI matrices go to results[c]
        (U_c * U_c floats each, in order).  Returns the number per sequence."""
        a = self._arrays(vis_re, vis_im, B, V, nb)
        count = a[-1]
        if len(sequence) != count:
            raise ValueError("one sequence index per snapshot")
        ns = len(self.sequences)
        seq = (ctypes.c_int * count)(*[int(c) for c in sequence])
        res = (ctypes.c_void_p * ns)(*[_ptr(r) if r is not None else None for r in results])
        nr = (ctypes.c_size_t * ns)()
        _check(lib().fip_batch_image_sequences(self._h, seq, *a, res, nr, _stream(stream)))
        return [int(x) for x in nr]

    def autotune(self, vis_re, vis_im, B, V, nb, stream=None) -> dict:
        _check(lib().fip_batch_autotune(self._h, *self._arrays(vis_re, vis_im, B, V, nb),
                                        _stream(stream)))
        return self.tuning()

    def autotune_sequences(self, sequence, vis_re, vis_im, B, V, nb, stream=None) -> list:
        """Autotunes on a representative call of several sequences; returns each
        sequence's tuning."""
        a = self._arrays(vis_re, vis_im, B, V, nb)
        seq = (ctypes.c_int * a[-1])(*[int(c) for c in sequence])
        _check(lib().fip_batch_autotune_sequences(self._h, seq, *a, _stream(stream)))
        return [self.tuning(c) for c in range(len(self.sequences))]

    def tuning(self, sequence: int = 0) -> dict:
        e, sp, dr, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().fip_batch_sequence_tuning(self._h, sequence, ctypes.byref(e),
                                               ctypes.byref(sp), ctypes.byref(dr),
                                               ctypes.byref(c)))
        return {"fft_values_per_thread": int(e.value), "fft_split": int(sp.value),
                "fft_direct": int(dr.value), "grid_ctas_per_sm": int(c.value)}

    def reset(self):
        _check(lib().fip_batch_reset(self._h))

    PHASES = ("prepare", "grid", "fft_cols", "fft_rows", "reproject", "trigger")

    def set_profiling(self, enable: bool):
        _check(lib().fip_batch_set_profiling(self._h, 1 if enable else 0))

    def phase_times(self) -> dict:
        """{phase: (total ms, calls)} of the profiled calls."""
        arr = (ctypes.c_double * len(self.PHASES))()
        calls = ctypes.c_long()
        _check(lib().fip_batch_phase_times(self._h, arr, len(self.PHASES), ctypes.byref(calls)))
        return {k: (arr[i], calls.value) for i, k in enumerate(self.PHASES)}

    def check(self, stream=None):
        """Raises FipError if a gather reprojection since the last check had a
        tile outside its domain (a folding wide-field geometry)."""
        _check(lib().fip_batch_check(self._h, _stream(stream)))

    @property
    def device_bytes(self) -> int:
        return int(lib().fip_batch_device_bytes(self._h))

    @property
    def kernel_launches(self) -> int:
        return int(lib().fip_batch_kernel_launches(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().fip_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def set_trigger_streaming(enable: bool) -> bool:
    """Plain-form sliding-window triggers (Imager.trigger_window, batches)
    stream every tile's slices through registers, each image read once (True,
    the default), or read each triple's three images (False); the tLISI is
    bit-identical either way.  Process-wide; returns the previous setting."""
    return bool(lib().fip_set_trigger_streaming(1 if enable else 0))


def grid_snapshot_noalloc(vis_re, vis_im, B, V, nb: int, image_size: int, cell_size: float,
                          grid, stream=None):
    """Gridding of one snapshot that allocates nothing (for callers that cannot
    allocate device memory): scratch in a fixed device array of the library;
    nb <= 131072, image_size <= 4096.  Output as Imager.grid_snapshot."""
    _check(lib().fip_grid_snapshot_noalloc(_ptr(vis_re), _ptr(vis_im), _ptr(B), _ptr(V), nb,
                                           image_size, float(cell_size), _ptr(grid),
                                           _stream(stream)))


def locate_transients(tlisi, image_size: int, unit_size: int, cell_size: float,
                      threshold: float = 0.99, max_out: int = 256, stream=None):
    """Transient locations from a device tLISI matrix (U*U floats): tiles below
    `threshold` that are the strict minimum of their 3 x 3 neighbourhood,
    refined to the neighbourhood's centroid of 1 - tLISI.  Returns
    (records, found): a LOCATION_DTYPE array of up to max_out locations,
    deepest first, and the number found."""
    out = np.zeros(max(int(max_out), 0), LOCATION_DTYPE)
    found = ctypes.c_size_t()
    _check(lib().fip_locate_transients(_ptr(tlisi), image_size, unit_size, float(cell_size),
                                       float(threshold), out.ctypes.data if out.size else None,
                                       out.size, ctypes.byref(found), _stream(stream)))
    return out[:min(found.value, out.size)], int(found.value)


def plane_project(uvw, freqs, rows: int, chans: int, B, V, stream=None):
    """Device plane fit: uvw [rows*3] m, freqs [chans] Hz -> B [rows*chans*2], V [9]."""
    _check(lib().fip_plane_project(_ptr(uvw), _ptr(freqs), rows, chans, _ptr(B), _ptr(V),
                                   _stream(stream)))


def collapse_visibilities(v0r, v0i, v3r, v3i, f0, f3, w0, w3, out_re, out_im, ns: int,
                          stream=None):
    _check(lib().fip_collapse_visibilities(*(_ptr(x) for x in (v0r, v0i, v3r, v3i, f0, f3, w0,
                                                               w3, out_re, out_im)), ns,
                                           _stream(stream)))


class Server:
    """Multi-beam streaming server (fip_server): continuous batching of
    snapshot requests, sliding-window tLISI per beam, HBM-budget admission."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 4, max_queue: int = 1024,
                 device: int = 0, max_step: int = None):
        h = ctypes.c_void_p()
        _check(lib().fip_server_create(ctypes.byref(h), device, int(hbm_budget_bytes), slots,
                                       max_queue))
        self._h = h
        self._beams = {}
        if max_step is not None:
            _check(lib().fip_server_set_max_step(self._h, int(max_step)))

    def stats(self) -> dict:
        """Merged launches run so far and the snapshots they imaged."""
        st, sn = ctypes.c_long(), ctypes.c_long()
        _check(lib().fip_server_stats(self._h, ctypes.byref(st), ctypes.byref(sn)))
        return {"steps": st.value, "snapshots": sn.value}

    def add_beam(self, image_size: int, max_baselines: int, cell_size: float, unit_size: int,
                 form: int = FORM_PLAIN, vis_storage: int = STORE_F32,
                 reproject: int = REPROJECT_GATHER) -> int:
        cfg = ImagerConfig(image_size, max_baselines, unit_size, cell_size, form, vis_storage, 0,
                           reproject)
        bid = ctypes.c_int()
        _check(lib().fip_server_add_beam(self._h, ctypes.byref(cfg), ctypes.byref(bid)))
        self._beams[bid.value] = (image_size // unit_size) ** 2
        return bid.value

    @property
    def reserved_bytes(self) -> int:
        return int(lib().fip_server_reserved_bytes(self._h))

    def submit(self, beam: int, vis_re, vis_im, B, V, nb: int) -> int:
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vis_re, vis_im, B, V)]
        rid = ctypes.c_long()
        _check(lib().fip_server_submit(self._h, beam, *(a.ctypes.data for a in arrs), nb,
                                       ctypes.byref(rid)))
        return rid.value

    def wait(self, request_id: int, timeout_ms: float = -1.0) -> dict:
        beam, seq, has = ctypes.c_int(), ctypes.c_long(), ctypes.c_int()
        lat = ctypes.c_double()
        n = max(self._beams.values()) if self._beams else 1
        buf = np.zeros(n, np.float32)
        _check(lib().fip_server_wait(self._h, request_id, timeout_ms, ctypes.byref(beam),
                                     ctypes.byref(seq), ctypes.byref(has), buf.ctypes.data, n,
                                     ctypes.byref(lat)))
        uu = self._beams[beam.value]
        u = int(round(uu ** 0.5))
        return {"beam": beam.value, "seq": seq.value, "latency_ms": lat.value,
                "tlisi": buf[:uu].reshape(u, u).copy() if has.value else None}

    def close(self):
        if getattr(self, "_h", None):
            lib().fip_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
