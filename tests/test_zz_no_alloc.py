"""agd_blend_device_noalloc: blending for callers that may not allocate device
memory (hosts whose memory pool owns the device, real-time code that must
not wait on or fail in the allocator).  It must give what agd_blend gives on the
same inputs, call after call, while keeping its intermediates in the
library's fixed device scratch array.  The device buffers here are made by
the test (torch) - the entry point itself allocates nothing.

This file is named to run after every other test file."""
import ctypes
from ctypes import POINTER, c_float, c_int, c_long, c_void_p

import numpy as np
import pytest

import agdeblend_b200 as A
from agdeblend_b200 import capi
from conftest import rel_l2
from problems import random_problem

pytestmark = pytest.mark.gpu

TOL = 1e-6  # the blend tests' tolerance (tests/test_gpu_deblend.py)


def _fn():
    lib = A.load_library(np.float32)
    fn = lib.agd_blend_device_noalloc
    ip, lp, fp = POINTER(c_int), POINTER(c_long), POINTER(c_float)
    fn.argtypes = [c_int, ip, ip, POINTER(lp), POINTER(ip), POINTER(ip), fp, c_int, c_int, c_int,
                   ip, ip, POINTER(lp), POINTER(ip), POINTER(ip), fp, c_void_p]
    fn.restype = c_int
    return fn


def _noalloc_blend(torch, shottimes, channels, trace_types, data, mode, taper, nt_out,
                   st_out, ch_out, tt_out):
    fn = _fn()
    nts = [d.shape[-1] for d in data]
    d_in = torch.from_numpy(np.concatenate([d.reshape(-1) for d in data]).astype(np.float32)).cuda()
    n_out = [int(np.asarray(s).size) for s in st_out]
    d_out = torch.full((sum(n * t for n, t in zip(n_out, nt_out)),), float("nan"),
                       dtype=torch.float32, device="cuda")
    keep = []

    def ints(v):
        a = np.ascontiguousarray(v, np.int32)
        keep.append(a)
        return a.ctypes.data_as(POINTER(c_int))

    def ptrs(arrs, dt, ct):
        p, k = capi._ptrs([np.asarray(a).reshape(-1) for a in arrs], dt, ct)
        keep.append(k)
        return p

    rc = fn(len(data), ints([int(np.asarray(s).size) for s in shottimes]), ints(nts),
            ptrs(shottimes, np.int64, c_long), ptrs(channels, np.int32, c_int),
            ptrs(trace_types, np.int32, c_int),
            ctypes.cast(d_in.data_ptr(), POINTER(c_float)), mode, taper, len(st_out),
            ints(n_out), ints(nt_out), ptrs(st_out, np.int64, c_long),
            ptrs(ch_out, np.int32, c_int), ptrs(tt_out, np.int32, c_int),
            ctypes.cast(d_out.data_ptr(), POINTER(c_float)), None)
    out = d_out.cpu().numpy()
    res, off = [], 0
    for n, t in zip(n_out, nt_out):
        res.append(out[off: off + n * t].reshape(n, t))
        off += n * t
    return rc, res


def _case(seed, mode, taper):
    sv = random_problem(seed, bad_missing=True)
    nts = [d.shape[-1] for d in sv.data]
    flat = [d.reshape(-1, n) for d, n in zip(sv.data, nts)]
    rng = np.random.default_rng(seed)
    st_out = [s + rng.integers(-3, 4, s.shape) for s in sv.shottimes]
    tt_out = [np.where(t == 1, 0, t).astype(np.int32) for t in sv.trace_types]
    nt_out = [n + 3 for n in nts]
    return sv, flat, st_out, tt_out, nt_out, mode, taper


def test_noalloc_blend_matches_agd_blend_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    for seed, mode, taper in [(1201, A.AGDBlendSum, 0), (1202, A.AGDBlendMean, 4),
                              (1203, A.AGDBlendOverwrite, 0)]:
        sv, flat, st_out, tt_out, nt_out, mode, taper = _case(seed, mode, taper)
        ref = A.blend(sv.shottimes, sv.channels, sv.trace_types, flat, mode,
                      taper_length=taper, n_times_out=nt_out, shottimes_out=st_out,
                      channels_out=sv.channels, trace_types_out=tt_out)
        rc, got = _noalloc_blend(torch, sv.shottimes, sv.channels, sv.trace_types, flat, mode,
                                 taper, nt_out, st_out, sv.channels, tt_out)
        assert rc == 0
        for g, r in zip(got, ref):
            assert np.isfinite(g).all()
            assert rel_l2(g, r.reshape(g.shape)) <= TOL


def test_noalloc_blend_rejects_oversized_problem(capfd):
    torch = pytest.importorskip("torch")
    n = 5_000_000  # a 20 MB record does not fit the 16 MiB scratch array
    fn = _fn()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    one = np.array([1], np.int32)
    nt = np.array([n], np.int32)
    st = np.array([0], np.int64)
    ch = np.array([0], np.int32)
    tt = np.array([0], np.int32)
    stp, k1 = capi._ptrs([st], np.int64, c_long)
    chp, k2 = capi._ptrs([ch], np.int32, c_int)
    ttp, k3 = capi._ptrs([tt], np.int32, c_int)
    p = ctypes.cast(buf.data_ptr(), POINTER(c_float))
    rc = fn(1, one.ctypes.data_as(POINTER(c_int)), nt.ctypes.data_as(POINTER(c_int)), stp, chp,
            ttp, p, A.AGDBlendSum, 0, 1, one.ctypes.data_as(POINTER(c_int)),
            nt.ctypes.data_as(POINTER(c_int)), stp, chp, ttp, p, None)
    assert rc == 1
    assert "16 MiB" in capfd.readouterr().err
