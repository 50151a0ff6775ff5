"""Test infrastructure only: ctypes bindings to the reference compiled by
oracle/Makefile into oracle/_ref/ (the reference's unchanged sources with the
project-written FFTW3 stand-in).

``RefOps`` wraps the operator harness (oracle/ref_ops.c) so the reference's
own model_forward / model_adjoint_update / blend_input / set_output run on
chosen inputs; ``ref_deblend`` / ``ref_blend`` call the reference library's
public agd_deblend / agd_blend.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_long, c_void_p

import numpy as np

from agdeblend_b200.capi import (DeblendArgs, bind_blend, bind_deblend, call_blend,
                                 call_deblend, real_ctype)

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")


def lib_path(name: str) -> str:
    return os.path.join(REF_DIR, name)


def available(name: str = "libagdeblend_refops.so") -> bool:
    return os.path.exists(lib_path(name))


_cache: dict = {}


def _load(name: str) -> ctypes.CDLL:
    if name not in _cache:
        _cache[name] = ctypes.CDLL(lib_path(name))
    return _cache[name]


class RefOps:
    """The reference's own operators on one problem (see oracle/ref_ops.c)."""

    def __init__(self, args: DeblendArgs):
        self.args = args
        self.dtype = args.dtype
        name = ("libagdeblend_refops_double.so" if self.dtype == np.float64
                else "libagdeblend_refops.so")
        lib = _load(name)
        rc = real_ctype(self.dtype)
        rp = POINTER(rc)
        self.lib = lib
        lib.refops_create.restype = c_void_p
        lib.refops_create.argtypes = bind_deblend(lib, self.dtype, "refops_create").argtypes[:12]
        lib.refops_create.restype = c_void_p
        lib.refops_destroy.argtypes = [c_void_p]
        lib.refops_n_windows.argtypes = [c_void_p]
        lib.refops_stepsize.argtypes = [c_void_p]
        lib.refops_stepsize.restype = c_double
        lib.refops_model_size.argtypes = [c_void_p]
        lib.refops_model_size.restype = c_long
        lib.refops_window_info.argtypes = [c_void_p, c_int, POINTER(c_int)]
        lib.refops_blended_layout.argtypes = [c_void_p, POINTER(c_long)]
        lib.refops_forward.argtypes = [c_void_p, rp, rp]
        lib.refops_adjoint.argtypes = [c_void_p, rp, rp]
        lib.refops_adjoint_update.argtypes = [c_void_p, rp, rc, rp]
        lib.refops_blend_input.argtypes = [c_void_p, POINTER(POINTER(c_int)),
                                           POINTER(rp), rp]
        lib.refops_set_output.argtypes = [c_void_p, rp, POINTER(rp)]
        lib.refops_initial_lamb.argtypes = [c_void_p, rp]
        lib.refops_initial_lamb.restype = c_double
        lib.refops_threshold.argtypes = [c_void_p, rp, rc]
        lib.refops_residual_norm.argtypes = [c_void_p, rp]
        lib.refops_residual_norm.restype = c_double
        self.h = lib.refops_create(*args.problem_args())
        if not self.h:
            raise RuntimeError("reference set_model failed")
        self._rp = rp
        self.n_windows = lib.refops_n_windows(self.h)
        self.model_size = int(lib.refops_model_size(self.h))
        nseg = lib.refops_blended_layout(self.h, None)
        seg = np.zeros(max(nseg, 1), np.int64)
        lib.refops_blended_layout(self.h, seg.ctypes.data_as(POINTER(c_long)))
        self.segments = seg[:nseg]
        self.record_size = int(self.segments.sum())
        self.stepsize = float(lib.refops_stepsize(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.refops_destroy(self.h)
            self.h = None

    def _p(self, a):
        return a.ctypes.data_as(self._rp)

    def window_info(self, w: int) -> np.ndarray:
        out = np.zeros(64, np.int32)
        self.lib.refops_window_info(self.h, w, out.ctypes.data_as(POINTER(c_int)))
        return out

    def forward(self, model: np.ndarray) -> np.ndarray:
        """model: interleaved real array of 2 * model_size."""
        m = np.ascontiguousarray(model, self.dtype)
        out = np.zeros(self.record_size, self.dtype)
        self.lib.refops_forward(self.h, self._p(m), self._p(out))
        return out

    def adjoint(self, record: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(record, self.dtype)
        out = np.zeros(2 * self.model_size, self.dtype)
        self.lib.refops_adjoint(self.h, self._p(r), self._p(out))
        return out

    def adjoint_update(self, record: np.ndarray, stepsize: float, model: np.ndarray):
        r = np.ascontiguousarray(record, self.dtype)
        m = np.array(model, self.dtype, copy=True)
        self.lib.refops_adjoint_update(self.h, self._p(r), stepsize, self._p(m))
        return m

    def blend_input(self, data: list) -> np.ndarray:
        from agdeblend_b200.capi import _ptrs
        d_p, keep = _ptrs([np.asarray(d).reshape(-1) for d in data], self.dtype,
                          real_ctype(self.dtype))
        out = np.zeros(self.record_size, self.dtype)
        rc = self.lib.refops_blend_input(self.h, self.args.shapes_p, d_p, self._p(out))
        if rc:
            raise RuntimeError("blend_input failed")
        return out

    def set_output(self, model: np.ndarray, shapes: list) -> list:
        from agdeblend_b200.capi import _ptrs
        m = np.ascontiguousarray(model, self.dtype)
        outs = [np.zeros(int(np.prod(s)), self.dtype) for s in shapes]
        o_p, keep = _ptrs(outs, self.dtype, real_ctype(self.dtype), writable=True)
        self.lib.refops_set_output(self.h, self._p(m), o_p)
        return [o.reshape(s) for o, s in zip(outs, shapes)]

    def initial_lamb(self, model: np.ndarray) -> float:
        m = np.ascontiguousarray(model, self.dtype)
        return float(self.lib.refops_initial_lamb(self.h, self._p(m)))

    def threshold(self, model: np.ndarray, lamb: float) -> np.ndarray:
        m = np.array(model, self.dtype, copy=True)
        self.lib.refops_threshold(self.h, self._p(m), lamb)
        return m

    def residual_norm(self, record: np.ndarray) -> float:
        r = np.ascontiguousarray(record, self.dtype)
        return float(self.lib.refops_residual_norm(self.h, self._p(r)))


def ref_deblend(args: DeblendArgs, initial_factor: float, n_its: int, print_freq: int = 0,
                lib_name: str | None = None) -> int:
    """The reference's public agd_deblend on ``args.data`` (in place)."""
    if lib_name is None:
        lib_name = ("libagdeblend_ref_double.so" if args.dtype == np.float64
                    else "libagdeblend_ref.so")
    fn = bind_deblend(_load(lib_name), args.dtype)
    return call_deblend(fn, args, initial_factor, n_its, print_freq)


def ref_blend(dtype, *blend_args, lib_name: str | None = None):
    if lib_name is None:
        lib_name = ("libagdeblend_ref_double.so" if np.dtype(dtype) == np.float64
                    else "libagdeblend_ref.so")
    fn = bind_blend(_load(lib_name), dtype)
    return call_blend(fn, dtype, *blend_args)
