"""AGDeblend on B200: Python host layer over the in-tree CUDA libraries.

``deblend`` and ``blend`` mirror the reference's Python wrapper
(wrappers/python/agdeblend/agdeblend.py:13-148 and :150-...) - same argument
names, meaning, defaults and errors - but call libagdeblend.so /
libagdeblend_double.so built from agdeblend_b200/csrc for sm_100a.
``Problem`` exposes the extension API (include/agdeblend_gpu.h): a planned
problem on which the operator, its adjoint and the solver can be applied
repeatedly.

There is no CPU fallback: if the CUDA library is missing the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_long, c_void_p

import numpy as np

from . import capi

AGDLive = 0
AGDBad = 1
AGDMissing = 2
AGDBlendSum = 0
AGDBlendMean = 1
AGDBlendOverwrite = 2

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAMES = {np.dtype(np.float32): "libagdeblend.so", np.dtype(np.float64): "libagdeblend_double.so"}
_libs: dict = {}


def library_path(dtype=np.float32) -> str:
    return os.path.join(PKG_DIR, LIB_NAMES[np.dtype(dtype)])


def load_library(dtype=np.float32) -> ctypes.CDLL:
    """Loads the CUDA library for ``dtype`` (float32 or float64)."""
    dtype = np.dtype(dtype)
    if dtype not in _libs:
        path = library_path(dtype)
        if not os.path.exists(path):
            raise RuntimeError(
                f"{os.path.basename(path)} is not built; run `python -m agdeblend_b200.build`")
        lib = ctypes.CDLL(path)
        _bind_extension(lib, dtype)
        _libs[dtype] = lib
    return _libs[dtype]


def _bind_extension(lib, dtype):
    rc = capi.real_ctype(dtype)
    rp = POINTER(rc)
    problem_args = capi.bind_deblend(lib, dtype, "agd_deblend").argtypes[:12]
    capi.bind_blend(lib, dtype, "agd_blend")
    lib.agd_gpu_problem_create.argtypes = problem_args + [POINTER(c_void_p)]
    lib.agd_gpu_problem_create.restype = c_int
    lib.agd_gpu_problem_destroy.argtypes = [c_void_p]
    lib.agd_gpu_problem_destroy.restype = None
    lib.agd_gpu_problem_info.argtypes = [c_void_p, POINTER(c_long)]
    lib.agd_gpu_problem_kernels.argtypes = [c_void_p, ctypes.c_char_p, c_int]
    lib.agd_gpu_stepsize.argtypes = [c_void_p, rp]
    lib.agd_gpu_forward.argtypes = [c_void_p, rp, rp]
    lib.agd_gpu_adjoint.argtypes = [c_void_p, rp, rp]
    lib.agd_gpu_blend_input.argtypes = [c_void_p, POINTER(rp), rp]
    lib.agd_gpu_set_output.argtypes = [c_void_p, rp, POINTER(rp)]
    lib.agd_gpu_solve.argtypes = [c_void_p, rc, c_int, c_int, POINTER(rp)]
    lib.agd_gpu_solve_range.argtypes = [c_void_p, rc, c_int, c_int, c_int, c_int, rp, rp,
                                        POINTER(rp)]
    lib.agd_gpu_time_iterations.argtypes = [c_void_p, POINTER(rp), rc, c_int, c_int, c_int,
                                            POINTER(c_double)]
    lib.agd_gpu_profile_iteration.argtypes = [c_void_p, rc, POINTER(c_double)]
    lib.agd_gpu_profile_iteration.restype = c_int
    lib.agd_plan_export.argtypes = problem_args + [POINTER(c_long), POINTER(c_int),
                                                   POINTER(c_long)]
    ip = POINTER(c_int)
    lip = POINTER(c_long)
    lib.agd_gpu_batch_create.argtypes = [
        c_int, ip, POINTER(ip), POINTER(ip), POINTER(POINTER(ip)), POINTER(POINTER(ip)),
        POINTER(POINTER(ip)), POINTER(POINTER(lip)), POINTER(POINTER(ip)), POINTER(POINTER(ip)),
        POINTER(ip), POINTER(POINTER(ip)), POINTER(POINTER(rp)), POINTER(c_void_p)]
    lib.agd_gpu_problem_steps.argtypes = [c_void_p, rp]
    lib.agd_gpu_problem_set_precision.argtypes = [c_void_p, c_int, POINTER(c_long)]
    for name in ("agd_gpu_problem_info", "agd_gpu_problem_kernels", "agd_gpu_stepsize", "agd_gpu_forward",
                 "agd_gpu_adjoint", "agd_gpu_blend_input", "agd_gpu_set_output",
                 "agd_gpu_solve", "agd_gpu_time_iterations", "agd_plan_export",
                 "agd_gpu_solve_range",
                 "agd_gpu_batch_create", "agd_gpu_problem_steps",
                 "agd_gpu_problem_set_precision"):
        getattr(lib, name).restype = c_int


def _dtype_of(data) -> np.dtype:
    d = np.asarray(data[0]).dtype
    if d == np.float64:
        return np.dtype(np.float64)
    if d == np.float32:
        return np.dtype(np.float32)
    raise RuntimeError("data must be float32 or float64")


def _n_dims(volumes, data):
    n_volumes = int(np.max(volumes)) + 1
    n_dims = np.zeros(n_volumes, np.int32)
    for v, d in zip(volumes, data):
        n_dims[int(v)] = np.asarray(d).ndim
    return n_dims


def _deblend_args(volumes, window_shapes, coords, shottimes, channels, trace_types, data,
                  wavelet_idxs=None, wavelets=None, dtype=None, in_place=False):
    """Checks and converts the arguments of ``deblend`` (the reference
    wrapper's, wrappers/python/agdeblend/agdeblend.py:71-146)."""
    dtype = _dtype_of(data) if dtype is None else np.dtype(dtype)
    if len(volumes) != len(data):
        raise RuntimeError("volumes must have the same length as data")
    for name, arr in (("coords", coords), ("shottimes", shottimes), ("channels", channels),
                      ("trace_types", trace_types)):
        if len(arr) != len(data):
            raise RuntimeError(f"{name} must have the same number of patches as data")
    n_traces = [int(np.prod(np.asarray(d).shape[:-1])) for d in data]
    for name, arr in (("shottimes", shottimes), ("channels", channels),
                      ("trace_types", trace_types)):
        for n, a in zip(n_traces, arr):
            if np.asarray(a).size != n:
                raise RuntimeError(f"{name} must have the same number of traces as data")
    if (wavelet_idxs is None) != (wavelets is None):
        raise RuntimeError("If wavelet_idxs or wavelets is not None, they both must not be")
    wavelet_lengths = None
    if wavelets is not None:
        wavelet_lengths = [len(w) for w in wavelets]
    shapes = [list(np.asarray(d).shape) for d in data]
    return capi.DeblendArgs(volumes, _n_dims(volumes, data), window_shapes, coords, shapes,
                            shottimes, channels, trace_types, data, wavelet_lengths,
                            wavelet_idxs, wavelets, dtype=dtype, in_place=in_place)


def deblend(volumes, window_shapes, coords, shottimes, channels, trace_types, initial_factor,
            n_its, print_freq, data, wavelet_idxs=None, wavelets=None, comm=None,
            overwrite_input=False):
    """Deblends seismic data; same arguments and result as the reference's
    ``agdeblend.deblend`` (serial form: ``comm`` must be None).  The input
    patches are left intact unless ``overwrite_input`` (an addition): then
    patches that are C-contiguous writable arrays of the data type are
    overwritten with the result and returned, with no copy, as the
    reference's wrapper does."""
    if comm is not None:
        raise RuntimeError("MPI communicators are not supported: the problem runs on one GPU")
    dtype = _dtype_of(data)
    lib = load_library(dtype)
    args = _deblend_args(volumes, window_shapes, coords, shottimes, channels, trace_types, data,
                         wavelet_idxs, wavelets, dtype, in_place=overwrite_input)
    fn = lib.agd_deblend
    if capi.call_deblend(fn, args, initial_factor, n_its, print_freq):
        raise RuntimeError("Error in call to agd_deblend")
    # args.data (this call's own copies of the input, or the input itself
    # with overwrite_input) hold the result: returned as they are (a second
    # copy would cost a full pass over the data)
    return args.data


def deblend_batch(problems, initial_factor, n_its):
    """Deblends independent problems together (agd_deblend_batch, an
    addition of this library).  ``problems``: one dict per problem with the
    keys of ``deblend`` (volumes, window_shapes, coords, shottimes, channels,
    trace_types, data, optionally wavelet_idxs and wavelets), all with the
    same data type.  Returns the deblended data of every problem, each as
    ``deblend`` would return it for that problem alone."""
    if not problems:
        return []
    dtype = _dtype_of(problems[0]["data"])
    lib = load_library(dtype)
    args = [_deblend_args(p["volumes"], p["window_shapes"], p["coords"], p["shottimes"],
                          p["channels"], p["trace_types"], p["data"], p.get("wavelet_idxs"),
                          p.get("wavelets"), dtype) for p in problems]
    batch = capi.BatchArgs(args)
    fn = capi.bind_deblend_batch(lib, dtype)
    if fn(*batch.problem_args(), initial_factor, n_its, batch.data_p):
        raise RuntimeError("Error in call to agd_deblend_batch")
    return [a.data for a in args]


def blend(shottimes, channels, trace_types, data, blend_mode, taper_length=0, n_times_out=None,
          shottimes_out=None, channels_out=None, trace_types_out=None, comm=None,
          data_out=None):
    """Blends seismic data or modifies already blended data; same arguments
    and result as the reference's ``agdeblend.blend`` (serial form)."""
    if comm is not None:
        raise RuntimeError("MPI communicators are not supported: the problem runs on one GPU")
    if blend_mode not in (AGDBlendSum, AGDBlendMean, AGDBlendOverwrite):
        raise RuntimeError("Invalid blend_mode")
    dtype = _dtype_of(data)
    lib = load_library(dtype)
    shottimes_out = shottimes if shottimes_out is None else shottimes_out
    channels_out = channels if channels_out is None else channels_out
    trace_types_out = trace_types if trace_types_out is None else trace_types_out
    n_times = [int(np.asarray(d).shape[-1]) for d in data]
    if data_out is not None:
        n_times_out = [int(np.asarray(d).shape[-1]) for d in data_out]
    elif n_times_out is None:
        n_times_out = n_times
    outs = None
    if data_out is not None:
        outs = [np.ascontiguousarray(d.reshape(-1, d.shape[-1])) for d in data_out]
        for d in outs:
            if d.dtype != dtype:
                raise RuntimeError("data_out does not have the right data type")
    rc, res = capi.call_blend(lib.agd_blend, dtype, n_times, shottimes, channels, trace_types,
                              [np.asarray(d).reshape(-1, n) for d, n in zip(data, n_times)],
                              blend_mode, taper_length, n_times_out, shottimes_out,
                              channels_out, trace_types_out, outs)
    if rc:
        raise RuntimeError("Error in call to agd_blend")
    shapes = [list(np.asarray(s).shape) + [n] for s, n in zip(shottimes_out, n_times_out)]
    if data_out is not None:
        for d, r in zip(data_out, res):
            d[...] = r.reshape(d.shape)
        return data_out
    return [r.reshape(s) for r, s in zip(res, shapes)]


class Problem:
    """A planned deblending problem on the current GPU (extension API)."""

    def __init__(self, volumes, n_dims, window_shapes, coords, shapes, shottimes, channels,
                 trace_types, wavelet_lengths=None, wavelet_idxs=None, wavelets=None,
                 dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self.lib = load_library(self.dtype)
        self.args = capi.DeblendArgs(volumes, n_dims, window_shapes, coords, shapes, shottimes,
                                     channels, trace_types, None, wavelet_lengths, wavelet_idxs,
                                     wavelets, dtype=self.dtype)
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        h = c_void_p()
        if self.lib.agd_gpu_problem_create(*self.args.problem_args(), ctypes.byref(h)):
            raise RuntimeError("agd_gpu_problem_create failed")
        self.h = h
        self._finish_init()

    @classmethod
    def from_batch(cls, surveys, dtype=np.float32):
        """A handle over independent problems solved together
        (agd_gpu_batch_create); its patches are all surveys' patches in
        order."""
        self = cls.__new__(cls)
        self.dtype = np.dtype(dtype)
        self.lib = load_library(self.dtype)
        self.sub_args = [capi.DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords,
                                          sv.shapes, sv.shottimes, sv.channels, sv.trace_types,
                                          None, sv.wavelet_lengths, sv.wavelet_idxs,
                                          sv.wavelets, dtype=self.dtype) for sv in surveys]
        self.args = capi.BatchArgs(self.sub_args)
        self.shapes = [tuple(int(v) for v in s) for sv in surveys for s in sv.shapes]
        h = c_void_p()
        if self.lib.agd_gpu_batch_create(*self.args.problem_args(), ctypes.byref(h)):
            raise RuntimeError("agd_gpu_batch_create failed")
        self.h = h
        self._finish_init()
        return self

    def _finish_init(self):
        info = np.zeros(23, np.int64)
        self.lib.agd_gpu_problem_info(self.h, info.ctypes.data_as(POINTER(c_long)))
        self.info = info
        self.n_windows = int(info[0])
        self.model_size = int(info[1])
        self.record_size = int(info[2])
        rc = capi.real_ctype(self.dtype)
        s = rc()
        self.lib.agd_gpu_stepsize(self.h, ctypes.byref(s))
        self.stepsize = float(s.value)
        self._rp = POINTER(rc)

    def kernels(self) -> dict:
        """Kernel family of each phase for the first window class and time
        group ({"space_fwd": ..., "space_adj": ..., "time_fwd": ...,
        "time_adj": ..., "wavelet": ...}), as profilers list the kernels."""
        buf = ctypes.create_string_buffer(512)
        self._check(self.lib.agd_gpu_problem_kernels(self.h, buf, len(buf)),
                    "agd_gpu_problem_kernels")
        return dict(kv.split("=", 1) for kv in buf.value.decode().split())

    PRECISION_FP32 = 0
    PRECISION_SPLIT_BF16 = 1

    def set_precision(self, mode: int) -> int:
        """Precision of the space DFTs (agd_gpu_problem_set_precision): 0
        FP32, 1 split-BF16 tensor-core contractions for windows of padded
        space shape 20 x 20 x 20.  Returns the number of windows the
        tensor-core kernels serve."""
        n = c_long(0)
        self._check(self.lib.agd_gpu_problem_set_precision(self.h, int(mode), ctypes.byref(n)),
                    "agd_gpu_problem_set_precision")
        return int(n.value)

    def steps(self) -> np.ndarray:
        """Step size of every problem of the handle."""
        n = len(getattr(self, "sub_args", [None]))
        out = np.zeros(n, self.dtype)
        self.lib.agd_gpu_problem_steps(self.h, out.ctypes.data_as(self._rp))
        return out

    @classmethod
    def from_survey(cls, sv, dtype=np.float32):
        return cls(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes, sv.shottimes,
                   sv.channels, sv.trace_types, sv.wavelet_lengths, sv.wavelet_idxs,
                   sv.wavelets, dtype=dtype)

    def close(self):
        if getattr(self, "h", None):
            self.lib.agd_gpu_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _p(self, a):
        return a.ctypes.data_as(self._rp)

    def _check(self, rc, name):
        if rc:
            raise RuntimeError(f"{name} failed")

    def forward(self, model: np.ndarray) -> np.ndarray:
        """A x; ``model`` interleaved (re, im) of 2 * model_size reals."""
        m = np.ascontiguousarray(model, self.dtype)
        out = np.zeros(self.record_size, self.dtype)
        self._check(self.lib.agd_gpu_forward(self.h, self._p(m), self._p(out)), "forward")
        return out

    def adjoint(self, record: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(record, self.dtype)
        out = np.zeros(2 * self.model_size, self.dtype)
        self._check(self.lib.agd_gpu_adjoint(self.h, self._p(r), self._p(out)), "adjoint")
        return out

    def _data_ptrs(self, data, writable=False, in_place=False):
        """Pointer array of patches; writable: arrays the call may overwrite -
        copies of the input, or with in_place the input patches themselves
        where they are C-contiguous writable arrays of the data type."""
        if writable and in_place:
            arrs = [np.require(d, self.dtype, ["C", "A", "W"]) for d in data]
        elif writable:
            arrs = [capi.private_copy(d, self.dtype) for d in data]
        else:
            arrs = [np.ascontiguousarray(d, self.dtype) for d in data]
        return capi._ptrs(arrs, self.dtype, capi.real_ctype(self.dtype), writable=writable)

    def blend_input(self, data) -> np.ndarray:
        ptrs, keep = self._data_ptrs(data)
        out = np.zeros(self.record_size, self.dtype)
        self._check(self.lib.agd_gpu_blend_input(self.h, ptrs, self._p(out)), "blend_input")
        return out

    def set_output(self, model: np.ndarray) -> list:
        m = np.ascontiguousarray(model, self.dtype)
        outs = [np.zeros(s, self.dtype) for s in self.shapes]
        ptrs, keep = capi._ptrs(outs, self.dtype, capi.real_ctype(self.dtype), writable=True)
        self._check(self.lib.agd_gpu_set_output(self.h, self._p(m), ptrs), "set_output")
        return outs

    def solve(self, data, initial_factor: float, n_its: int, print_freq: int = 0,
              overwrite_input: bool = False) -> list:
        """agd_gpu_solve: the deblended patches (with overwrite_input, written
        over the input patches where they are C-contiguous writable arrays
        of the data type, as deblend(..., overwrite_input=True))."""
        ptrs, keep = self._data_ptrs(data, writable=True, in_place=overwrite_input)
        self._check(self.lib.agd_gpu_solve(self.h, initial_factor, n_its, print_freq, ptrs),
                    "solve")
        return [k.reshape(s) for k, s in zip(keep, self.shapes)]

    def solve_range(self, data, initial_factor: float, n_its: int, it_begin: int, it_end: int,
                    model_in=None, print_freq: int = 0):
        """Iterations [it_begin, it_end) of the n_its schedule (checkpoint /
        resume).  Returns (output patches, model after iteration it_end - 1)."""
        ptrs, keep = self._data_ptrs(data, writable=True)
        m_in = None
        if model_in is not None:
            m_in = np.ascontiguousarray(model_in, self.dtype)
        m_out = np.zeros(2 * self.model_size, self.dtype)
        self._check(self.lib.agd_gpu_solve_range(
            self.h, initial_factor, n_its, it_begin, it_end, print_freq,
            self._p(m_in) if m_in is not None else None, self._p(m_out), ptrs), "solve_range")
        return [k.reshape(s) for k, s in zip(keep, self.shapes)], m_out

    def time_iterations(self, data, initial_factor: float, n_its: int, warmup: int,
                        steps: int) -> np.ndarray:
        ptrs, keep = self._data_ptrs(data)
        t = np.zeros(4, np.float64)
        self._check(self.lib.agd_gpu_time_iterations(
            self.h, ptrs, initial_factor, n_its, warmup, steps,
            t.ctypes.data_as(POINTER(c_double))), "time_iterations")
        return t

    def profile_iteration(self, lamb: float) -> np.ndarray:
        ms = np.zeros(16, np.float64)
        self._check(self.lib.agd_gpu_profile_iteration(
            self.h, lamb, ms.ctypes.data_as(POINTER(c_double))), "profile_iteration")
        return ms


def plan_export(volumes, n_dims, window_shapes, coords, shapes, shottimes, channels,
                trace_types, wavelet_lengths=None, wavelet_idxs=None, wavelets=None,
                dtype=np.float32):
    """Host planning only (no GPU): (info[8], windows[n, 32], blend[n_traces, 3])."""
    lib = load_library(dtype)
    args = capi.DeblendArgs(volumes, n_dims, window_shapes, coords, shapes, shottimes, channels,
                            trace_types, None, wavelet_lengths, wavelet_idxs, wavelets,
                            dtype=dtype)
    info = np.zeros(8, np.int64)
    if lib.agd_plan_export(*args.problem_args(), info.ctypes.data_as(POINTER(c_long)), None,
                           None):
        raise RuntimeError("agd_plan_export failed")
    win = np.zeros((int(info[0]), 32), np.int32)
    blend_c = np.zeros((int(info[3]), 3), np.int64)
    lib.agd_plan_export(*args.problem_args(), info.ctypes.data_as(POINTER(c_long)),
                        win.ctypes.data_as(POINTER(c_int)), blend_c.ctypes.data_as(POINTER(c_long)))
    return info, win, blend_c
