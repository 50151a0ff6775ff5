"""agd_blend_device_noalloc: blending for callers that may not allocate device
memory (hosts whose memory pool owns the device, real-time code that must
not wait on or fail in the allocator).  It must give what agd_blend and the
float64 oracle's blend give on the same inputs, call after call, while
keeping its intermediates in the library's fixed 16 MiB device scratch
array; it must accept a problem whose tables just fit that array and reject
one that just does not.  The device buffers here are made by the test
(torch) - the entry point itself allocates nothing.

This file is named to run after every other test file."""
import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_long, c_void_p

import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import capi
from conftest import rel_l2
from problems import random_problem

pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-6, np.float64: 1e-12}  # the blend tests' tolerances
SCRATCH_BYTES = 16 << 20


def _fn(dtype):
    lib = A.load_library(dtype)
    fn = lib.agd_blend_device_noalloc
    rp = POINTER(c_float if dtype == np.float32 else c_double)
    ip, lp = POINTER(c_int), POINTER(c_long)
    fn.argtypes = [c_int, ip, ip, POINTER(lp), POINTER(ip), POINTER(ip), rp, c_int, c_int, c_int,
                   ip, ip, POINTER(lp), POINTER(ip), POINTER(ip), rp, c_void_p]
    fn.restype = c_int
    return fn, rp


def _noalloc_blend(torch, shottimes, channels, trace_types, data, mode, taper, nt_out,
                   st_out, ch_out, tt_out, dtype=np.float32, stream=None):
    fn, rp = _fn(dtype)
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    nts = [d.shape[-1] for d in data]
    d_in = torch.from_numpy(np.concatenate([d.reshape(-1) for d in data]).astype(dtype)).cuda()
    n_out = [int(np.asarray(s).size) for s in st_out]
    d_out = torch.full((sum(n * t for n, t in zip(n_out, nt_out)),), float("nan"), dtype=tdt,
                       device="cuda")
    keep = []

    def ints(v):
        a = np.ascontiguousarray(v, np.int32)
        keep.append(a)
        return a.ctypes.data_as(POINTER(c_int))

    def ptrs(arrs, dt, ct):
        p, k = capi._ptrs([np.asarray(a).reshape(-1) for a in arrs], dt, ct)
        keep.append(k)
        return p

    handle = None
    if stream is not None:
        # the inputs were written on torch's current stream
        stream.wait_stream(torch.cuda.current_stream())
        handle = c_void_p(stream.cuda_stream)
    rc = fn(len(data), ints([int(np.asarray(s).size) for s in shottimes]), ints(nts),
            ptrs(shottimes, np.int64, c_long), ptrs(channels, np.int32, c_int),
            ptrs(trace_types, np.int32, c_int), ctypes.cast(d_in.data_ptr(), rp), mode, taper,
            len(st_out), ints(n_out), ints(nt_out), ptrs(st_out, np.int64, c_long),
            ptrs(ch_out, np.int32, c_int), ptrs(tt_out, np.int32, c_int),
            ctypes.cast(d_out.data_ptr(), rp), handle)
    out = d_out.cpu().numpy()
    res, off = [], 0
    for n, t in zip(n_out, nt_out):
        res.append(out[off: off + n * t].reshape(n, t))
        off += n * t
    return rc, res


def _case(seed, mode, taper, dtype=np.float32):
    sv = random_problem(seed, bad_missing=True)
    nts = [d.shape[-1] for d in sv.data]
    flat = [d.reshape(-1, n).astype(dtype) for d, n in zip(sv.data, nts)]
    rng = np.random.default_rng(seed)
    st_out = [s + rng.integers(-3, 4, s.shape) for s in sv.shottimes]
    tt_out = [np.where(t == 1, 0, t).astype(np.int32) for t in sv.trace_types]
    nt_out = [n + 3 for n in nts]
    return sv, flat, st_out, tt_out, nt_out, mode, taper


CASES = [(1201, A.AGDBlendSum, 0), (1202, A.AGDBlendMean, 4), (1203, A.AGDBlendOverwrite, 0)]


def test_noalloc_blend_matches_agd_blend_and_oracle_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    for seed, mode, taper in CASES:
        sv, flat, st_out, tt_out, nt_out, mode, taper = _case(seed, mode, taper)
        nts = [f.shape[-1] for f in flat]
        ref = A.blend(sv.shottimes, sv.channels, sv.trace_types, flat, mode,
                      taper_length=taper, n_times_out=nt_out, shottimes_out=st_out,
                      channels_out=sv.channels, trace_types_out=tt_out)
        ora = O.blend(nts, sv.shottimes, sv.channels, sv.trace_types, flat, mode, taper, nt_out,
                      st_out, sv.channels, tt_out)
        rc, got = _noalloc_blend(torch, sv.shottimes, sv.channels, sv.trace_types, flat, mode,
                                 taper, nt_out, st_out, sv.channels, tt_out)
        assert rc == 0
        for g, r, o in zip(got, ref, ora):
            assert np.isfinite(g).all()
            assert rel_l2(g, r.reshape(g.shape)) <= TOL[np.float32]
            assert rel_l2(g, np.asarray(o).reshape(g.shape)) <= TOL[np.float32]


def test_noalloc_blend_double_library_on_a_caller_stream():
    torch = pytest.importorskip("torch")
    stream = torch.cuda.Stream()
    for seed, mode, taper in CASES[:2]:
        sv, flat, st_out, tt_out, nt_out, mode, taper = _case(seed + 10, mode, taper,
                                                              np.float64)
        nts = [f.shape[-1] for f in flat]
        ora = O.blend(nts, sv.shottimes, sv.channels, sv.trace_types, flat, mode, taper, nt_out,
                      st_out, sv.channels, tt_out)
        rc, got = _noalloc_blend(torch, sv.shottimes, sv.channels, sv.trace_types, flat, mode,
                                 taper, nt_out, st_out, sv.channels, tt_out, np.float64, stream)
        assert rc == 0
        for g, o in zip(got, ora):
            assert rel_l2(g, np.asarray(o).reshape(g.shape)) <= TOL[np.float64]


def _align(v):
    return (v + 255) & ~255


def _scratch_bytes_one_trace(n):
    """Scratch the entry point carves for one float trace of n samples blended
    into one channel and read back once: the record, the chunk CSR (512
    samples per chunk), one contribution (24 bytes) per chunk, the mute mask
    and the five per-output-trace tables, each region 256-byte aligned."""
    n_chunk = (n + 511) // 512
    off = _align(4 * n)
    off = _align(off + 8 * (n_chunk + 1))
    off = _align(off + 24 * n_chunk)
    off = _align(off + n)
    for size in (8, 8, 4, 4, 4):
        off = _align(off + size)
    return off


def _largest_fitting_trace():
    lo, hi = 1, SCRATCH_BYTES
    while lo < hi:  # largest n whose scratch fits
        mid = (lo + hi + 1) // 2
        if _scratch_bytes_one_trace(mid) <= SCRATCH_BYTES:
            lo = mid
        else:
            hi = mid - 1
    return lo


def _one_trace_call(torch, n):
    rng = np.random.default_rng(n)
    trace = rng.standard_normal((1, n)).astype(np.float32)
    st = [np.array([5], np.int64)]
    ch = [np.array([3], np.int32)]
    tt = [np.array([0], np.int32)]
    return trace, _noalloc_blend(torch, st, ch, tt, [trace], A.AGDBlendSum, 0, [n], st, ch, tt)


def test_noalloc_blend_size_limit_boundary(capfd):
    torch = pytest.importorskip("torch")
    n = _largest_fitting_trace()
    assert _scratch_bytes_one_trace(n) <= SCRATCH_BYTES < _scratch_bytes_one_trace(n + 1)
    assert n > 3_000_000
    trace, (rc, got) = _one_trace_call(torch, n)
    assert rc == 0
    assert np.array_equal(got[0], trace)  # one trace summed alone reads back unchanged
    # the next sample no longer fits: rejected before any device work
    _, (rc, got) = _one_trace_call(torch, n + 1)
    assert rc == 1
    assert "16 MiB" in capfd.readouterr().err
    assert np.isnan(got[0]).all()


def test_noalloc_blend_rejects_oversized_problem(capfd):
    torch = pytest.importorskip("torch")
    n = 5_000_000  # a 20 MB record does not fit the 16 MiB scratch array
    fn, _ = _fn(np.float32)
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
