"""ctypes marshalling for libraries that export the AGDeblend C API.

``agd_deblend`` and ``agd_blend`` take arrays of per-patch pointers
(include/agdeblend.h:22-44 of the reference).  ``DeblendArgs`` builds those
pointer arrays from per-patch numpy arrays and keeps the buffers alive for the
duration of the call, the same conversion the reference's cffi wrapper does
(wrappers/python/agdeblend/agdeblend.py:71-146).
"""
from __future__ import annotations

import ctypes
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from ctypes import POINTER, c_double, c_float, c_int, c_long, c_void_p

import numpy as np

_COPY_THREADS_MIN_BYTES = 16 << 20
_COPY_WORKERS = max(1, min(16, os.cpu_count() or 1))
_copy_pool = None
_copy_pool_lock = threading.Lock()


def _pool() -> ThreadPoolExecutor:
    global _copy_pool
    with _copy_pool_lock:
        if _copy_pool is None:
            _copy_pool = ThreadPoolExecutor(max_workers=_COPY_WORKERS)
        return _copy_pool


def private_copy(d, dtype) -> np.ndarray:
    """A C-ordered copy of ``d`` in ``dtype`` that the library may overwrite.
    Large contiguous arrays already of ``dtype`` are copied in parallel
    slices (numpy releases the GIL while copying), which matters for the
    hundreds of megabytes of a 4-D survey."""
    a = np.asarray(d)
    if a.dtype != dtype or not a.flags.c_contiguous or a.nbytes < _COPY_THREADS_MIN_BYTES:
        return np.array(a, dtype=dtype, order="C", copy=True)
    out = np.empty(a.shape, dtype)
    src, dst = a.reshape(-1), out.reshape(-1)
    pool = _pool()
    n = _COPY_WORKERS
    step = (src.size + n - 1) // n
    list(pool.map(lambda i: np.copyto(dst[i * step:(i + 1) * step], src[i * step:(i + 1) * step]),
                  range(n)))
    return out

_c_int_p = POINTER(c_int)
_c_long_p = POINTER(c_long)


def real_ctype(dtype) -> type:
    return c_double if np.dtype(dtype) == np.float64 else c_float


def _ptrs(arrays, np_dtype, ctype, writable=False):
    keep = []
    for a in arrays:
        if writable:
            if not (isinstance(a, np.ndarray) and a.dtype == np_dtype and a.flags.c_contiguous):
                raise TypeError("writable patch arrays must be C-contiguous " + str(np_dtype))
            keep.append(a)
        else:
            keep.append(np.ascontiguousarray(a, dtype=np_dtype))
    arr = (POINTER(ctype) * max(len(keep), 1))()
    for i, a in enumerate(keep):
        arr[i] = a.ctypes.data_as(POINTER(ctype))
    return arr, keep


def _vec(values, np_dtype, ctype):
    a = np.ascontiguousarray(values, dtype=np_dtype)
    return a.ctypes.data_as(POINTER(ctype)), a


def bind_deblend(lib: ctypes.CDLL, dtype, name: str = "agd_deblend"):
    fn = getattr(lib, name)
    rc = real_ctype(dtype)
    fn.restype = c_int
    fn.argtypes = [c_int, _c_int_p, _c_int_p, POINTER(_c_int_p), POINTER(_c_int_p),
                   POINTER(_c_int_p), POINTER(_c_long_p), POINTER(_c_int_p),
                   POINTER(_c_int_p), _c_int_p, POINTER(_c_int_p),
                   POINTER(POINTER(rc)), rc, c_int, c_int, POINTER(POINTER(rc))]
    return fn


def bind_blend(lib: ctypes.CDLL, dtype, name: str = "agd_blend"):
    fn = getattr(lib, name)
    rc = real_ctype(dtype)
    fn.restype = c_int
    fn.argtypes = [c_int, _c_int_p, _c_int_p, POINTER(_c_long_p), POINTER(_c_int_p),
                   POINTER(_c_int_p), POINTER(POINTER(rc)), c_int, c_int, c_int,
                   _c_int_p, _c_int_p, POINTER(_c_long_p), POINTER(_c_int_p),
                   POINTER(_c_int_p), POINTER(POINTER(rc))]
    return fn


class DeblendArgs:
    """Pointer-array form of agd_deblend's problem description.  ``data`` is
    converted to writable ``dtype`` arrays (the call overwrites them)."""

    def __init__(self, volumes, n_dims, window_shapes, coords, shapes, shottimes,
                 channels, trace_types, data=None, wavelet_lengths=None,
                 wavelet_idxs=None, wavelets=None, dtype=np.float32, in_place=False):
        self.dtype = np.dtype(dtype)
        rc = real_ctype(dtype)
        self.n_patches = len(volumes)
        self.volumes_p, self._v = _vec(volumes, np.int32, c_int)
        self.n_dims_p, self._nd = _vec(n_dims, np.int32, c_int)
        self.window_shapes_p, self._ws = _ptrs(window_shapes, np.int32, c_int)
        coords_fixed = [c if len(c) else [0] for c in coords]
        self.coords_p, self._co = _ptrs(coords_fixed, np.int32, c_int)
        self.shapes_p, self._sh = _ptrs(shapes, np.int32, c_int)
        self.shottimes_p, self._st = _ptrs([np.asarray(s).reshape(-1) for s in shottimes],
                                           np.int64, c_long)
        self.channels_p, self._ch = _ptrs([np.asarray(c).reshape(-1) for c in channels],
                                          np.int32, c_int)
        self.trace_types_p, self._tt = _ptrs([np.asarray(t).reshape(-1) for t in trace_types],
                                             np.int32, c_int)
        if wavelet_lengths is not None:
            self.wavelet_lengths_p, self._wl = _vec(wavelet_lengths, np.int32, c_int)
            self.wavelet_idxs_p, self._wi = _ptrs(
                [np.asarray(w).reshape(-1) for w in wavelet_idxs], np.int32, c_int)
            self.wavelets_p, self._wv = _ptrs(wavelets, self.dtype, rc)
        else:
            self.wavelet_lengths_p = None
            self.wavelet_idxs_p = None
            self.wavelets_p = None
        self.data = None
        if data is not None:
            self.set_data(data, in_place)

    def set_data(self, data, in_place=False):
        """in_place: arrays that are already C-contiguous, aligned, writable
        ``dtype`` arrays are used as they are (the call overwrites them, as
        the reference's own wrapper does); others are copied."""
        if in_place:
            self.data = [np.require(d, self.dtype, ["C", "A", "W"]) for d in data]
        else:
            self.data = [private_copy(d, self.dtype) for d in data]
        self.data_p, _ = _ptrs(self.data, self.dtype, real_ctype(self.dtype), writable=True)

    def problem_args(self):
        """The 12 leading arguments shared by agd_deblend and the planning
        entry points (n_patches ... wavelets)."""
        return (self.n_patches, self.volumes_p, self.n_dims_p, self.window_shapes_p,
                self.coords_p, self.shapes_p, self.shottimes_p, self.channels_p,
                self.trace_types_p, self.wavelet_lengths_p, self.wavelet_idxs_p,
                self.wavelets_p)


def call_deblend(fn, args: DeblendArgs, initial_factor: float, n_its: int,
                 print_freq: int = 0) -> int:
    return fn(*args.problem_args(), initial_factor, n_its, print_freq, args.data_p)


def call_blend(fn, dtype, n_times, shottimes, channels, trace_types, data, blend_mode,
               taper_length, n_times_out, shottimes_out, channels_out, trace_types_out,
               data_out=None):
    """Calls an agd_blend-compatible function.  Returns (rc, data_out list)."""
    dtype = np.dtype(dtype)
    rc_t = real_ctype(dtype)
    n_patches = len(shottimes)
    n_traces = [int(np.asarray(s).size) for s in shottimes]
    n_traces_out = [int(np.asarray(s).size) for s in shottimes_out]
    nt_p, k1 = _vec(n_traces, np.int32, c_int)
    ntm_p, k2 = _vec(n_times, np.int32, c_int)
    st_p, k3 = _ptrs([np.asarray(s).reshape(-1) for s in shottimes], np.int64, c_long)
    ch_p, k4 = _ptrs([np.asarray(s).reshape(-1) for s in channels], np.int32, c_int)
    tt_p, k5 = _ptrs([np.asarray(s).reshape(-1) for s in trace_types], np.int32, c_int)
    dat = [np.ascontiguousarray(np.asarray(d, dtype=dtype)) for d in data]
    d_p, k6 = _ptrs(dat, dtype, rc_t, writable=True)
    nto_p, k7 = _vec(n_traces_out, np.int32, c_int)
    ntmo_p, k8 = _vec(n_times_out, np.int32, c_int)
    sto_p, k9 = _ptrs([np.asarray(s).reshape(-1) for s in shottimes_out], np.int64, c_long)
    cho_p, k10 = _ptrs([np.asarray(s).reshape(-1) for s in channels_out], np.int32, c_int)
    tto_p, k11 = _ptrs([np.asarray(s).reshape(-1) for s in trace_types_out], np.int32, c_int)
    if data_out is None:
        data_out = [np.zeros((n, t), dtype) for n, t in zip(n_traces_out, n_times_out)]
    do_p, k12 = _ptrs(data_out, dtype, rc_t, writable=True)
    rc = fn(n_patches, nt_p, ntm_p, st_p, ch_p, tt_p, d_p, blend_mode, taper_length,
            len(shottimes_out), nto_p, ntmo_p, sto_p, cho_p, tto_p, do_p)
    return rc, data_out


def bind_deblend_batch(lib: ctypes.CDLL, dtype, name: str = "agd_deblend_batch"):
    """agd_deblend_batch (include/agdeblend_gpu.h): every argument an array
    over the problems of the agd_deblend argument."""
    fn = getattr(lib, name)
    rc = real_ctype(dtype)
    rp = POINTER(rc)
    fn.restype = c_int
    fn.argtypes = [c_int, _c_int_p, POINTER(_c_int_p), POINTER(_c_int_p),
                   POINTER(POINTER(_c_int_p)), POINTER(POINTER(_c_int_p)),
                   POINTER(POINTER(_c_int_p)), POINTER(POINTER(_c_long_p)),
                   POINTER(POINTER(_c_int_p)), POINTER(POINTER(_c_int_p)), POINTER(_c_int_p),
                   POINTER(POINTER(_c_int_p)), POINTER(POINTER(rp)), rc, c_int,
                   POINTER(POINTER(rp))]
    return fn


class BatchArgs:
    """Per-problem DeblendArgs gathered into the pointer arrays of
    agd_deblend_batch / agd_gpu_batch_create."""

    def __init__(self, problems):
        self.problems = list(problems)
        n = len(self.problems)
        self.dtype = self.problems[0].dtype
        rc = real_ctype(self.dtype)
        rp = POINTER(rc)
        self.n_problems = n
        self.n_patches_p, self._np = _vec([a.n_patches for a in self.problems], np.int32, c_int)

        def arr(ctype, values):
            a = (ctype * max(n, 1))()
            for i, v in enumerate(values):
                a[i] = ctypes.cast(v, ctype) if v is not None else ctype()
            return a

        P = self.problems
        self.volumes_p = arr(_c_int_p, [a.volumes_p for a in P])
        self.n_dims_p = arr(_c_int_p, [a.n_dims_p for a in P])
        self.window_shapes_p = arr(POINTER(_c_int_p), [a.window_shapes_p for a in P])
        self.coords_p = arr(POINTER(_c_int_p), [a.coords_p for a in P])
        self.shapes_p = arr(POINTER(_c_int_p), [a.shapes_p for a in P])
        self.shottimes_p = arr(POINTER(_c_long_p), [a.shottimes_p for a in P])
        self.channels_p = arr(POINTER(_c_int_p), [a.channels_p for a in P])
        self.trace_types_p = arr(POINTER(_c_int_p), [a.trace_types_p for a in P])
        if any(a.wavelets_p is not None for a in P):
            self.wavelet_lengths_p = arr(_c_int_p, [a.wavelet_lengths_p for a in P])
            self.wavelet_idxs_p = arr(POINTER(_c_int_p), [a.wavelet_idxs_p for a in P])
            self.wavelets_p = arr(POINTER(rp), [a.wavelets_p for a in P])
        else:
            self.wavelet_lengths_p = self.wavelet_idxs_p = self.wavelets_p = None
        if all(a.data is not None for a in P):
            self.data_p = arr(POINTER(rp), [a.data_p for a in P])
        else:
            self.data_p = None

    def problem_args(self):
        """The 13 leading arguments of agd_deblend_batch / agd_gpu_batch_create."""
        return (self.n_problems, self.n_patches_p, self.volumes_p, self.n_dims_p,
                self.window_shapes_p, self.coords_p, self.shapes_p, self.shottimes_p,
                self.channels_p, self.trace_types_p, self.wavelet_lengths_p,
                self.wavelet_idxs_p, self.wavelets_p)
