"""Input validation of agd_deblend / agd_blend (CPU only: every case fails
before any device work).  Each case is a branch of the reference's
check_deblend_inputs (src/agdeblend.c:263-509) or check_blend_inputs
(src/agdeblend.c:651-732); the call must return 1 and print the reference's
message to stderr."""
import numpy as np
import pytest

import agdeblend_b200 as A
from agdeblend_b200 import capi
from agdeblend_b200 import synthetic as S


def _args(sv, **over):
    kw = dict(volumes=sv.volumes, n_dims=sv.n_dims, window_shapes=sv.window_shapes,
              coords=sv.coords, shapes=sv.shapes, shottimes=sv.shottimes,
              channels=sv.channels, trace_types=sv.trace_types, data=sv.data,
              wavelet_lengths=sv.wavelet_lengths, wavelet_idxs=sv.wavelet_idxs,
              wavelets=sv.wavelets)
    kw.update(over)
    return capi.DeblendArgs(**kw)


def _call(args, initial_factor=1.0, n_its=10, n_patches=None, null=()):
    lib = A.load_library(np.float32)
    a = list(args.problem_args())
    names = ["n_patches", "volumes", "n_dims", "window_shapes", "coords", "shapes",
             "shottimes", "channels", "trace_types", "wavelet_lengths", "wavelet_idxs",
             "wavelets"]
    for n in null:
        if n != "data":
            a[names.index(n)] = None
    if n_patches is not None:
        a[0] = n_patches
    return lib.agd_deblend(*a, initial_factor, n_its, 0, None if "data" in null else args.data_p)


@pytest.fixture(scope="module")
def sv():
    return S.gather_2d(seed=3, n_shots=32, nt=128, window=(16, 64))


@pytest.mark.parametrize("kwargs,msg", [
    (dict(n_patches=0), "n_patches must be > 0"),
    (dict(n_its=0), "n_its must be > 0"),
    (dict(initial_factor=0.0), "initial_factor must be in (0, 1]"),
    (dict(initial_factor=1.5), "initial_factor must be in (0, 1]"),
    (dict(null=("volumes",)), "volumes must not be NULL"),
    (dict(null=("n_dims",)), "n_dims must not be NULL"),
    (dict(null=("window_shapes",)), "window_shapes must not be NULL"),
    (dict(null=("coords",)), "coords must not be NULL"),
    (dict(null=("shapes",)), "shapes must not be NULL"),
    (dict(null=("shottimes",)), "shottimes must not be NULL"),
    (dict(null=("channels",)), "channels must not be NULL"),
    (dict(null=("trace_types",)), "trace_types must not be NULL"),
    (dict(null=("data",)), "data must not be NULL"),
])
def test_deblend_rejects(sv, capfd, kwargs, msg):
    assert _call(_args(sv), **kwargs) == 1
    err = capfd.readouterr().err
    assert msg in err and "ERROR in agd_deblend" in err


@pytest.mark.parametrize("over,msg", [
    (dict(n_dims=[1]), "n_dims must be > 1"),
    (dict(window_shapes=[[1, 64]]), "window_shapes must be at least 2"),
    (dict(window_shapes=[[15, 64]]), "window_shapes must be even"),
    (dict(window_shapes=[[64, 64]]), "window_shape must not be bigger than patch shape"),
])
def test_deblend_rejects_shapes(sv, capfd, over, msg):
    assert _call(_args(sv, **over)) == 1
    assert msg in capfd.readouterr().err


def test_deblend_rejects_too_many_dims(capfd):
    sv = S.gather_2d(seed=3, n_shots=32, nt=128, window=(16, 64))
    args = _args(sv, n_dims=[6], window_shapes=[[2, 2, 2, 2, 2, 64]],
                 shapes=[[2, 2, 2, 2, 2, 128]], coords=[[0] * 5])
    assert _call(args) == 1
    assert "AGD_MAX_N_COORDS" in capfd.readouterr().err


def test_deblend_rejects_partial_wavelets(sv, capfd):
    args = _args(sv, wavelet_lengths=[4], wavelet_idxs=[np.zeros(32, np.int32)],
                 wavelets=[np.ones(4, np.float32)])
    assert _call(args, null=("wavelets",)) == 1
    assert "wavelets must not be NULL" in capfd.readouterr().err


def test_deblend_rejects_negative_wavelet_index(sv, capfd):
    idx = np.zeros(32, np.int32)
    idx[3] = -1
    args = _args(sv, wavelet_lengths=[4], wavelet_idxs=[idx], wavelets=[np.ones(4, np.float32)])
    assert _call(args) == 1
    assert "wavelet_idx must not be negative" in capfd.readouterr().err


def test_deblend_rejects_mixed_wavelet_lengths(sv, capfd):
    idx = np.zeros(32, np.int32)
    idx[5] = 1
    args = _args(sv, wavelet_lengths=[4, 5], wavelet_idxs=[idx],
                 wavelets=[np.ones(4, np.float32), np.ones(5, np.float32)])
    assert _call(args) == 1
    assert "same length" in capfd.readouterr().err


def test_deblend_rejects_odd_tapered_window(capfd):
    """Two neighbouring patches with an odd window that equals the patch
    width: the shared edge would be tapered (src/model.c:551-580)."""
    rng = np.random.default_rng(0)
    shapes = [[9, 64], [9, 64]]
    st = [np.arange(9, dtype=np.int64) * 50, 500 + np.arange(9, dtype=np.int64) * 50]
    sv = S.Survey("odd", [0, 0], [2], [[9, 32]], [[0], [1]], shapes, st,
                  [np.zeros(9, np.int32)] * 2, [np.zeros(9, np.int32)] * 2,
                  [rng.standard_normal((9, 64)).astype(np.float32) for _ in range(2)],
                  [None, None], 5)
    assert _call(_args(sv)) == 1
    assert "may only be odd if there is no tapering" in capfd.readouterr().err


def _blend(n_patches=1, taper=0, mode=A.AGDBlendSum, out_types=None, null_data=False):
    lib = A.load_library(np.float32)
    st = [np.arange(4, dtype=np.int64) * 3]
    ch = [np.zeros(4, np.int32)]
    tt = [np.zeros(4, np.int32)]
    data = [np.ones((4, 5), np.float32)]
    tto = out_types if out_types is not None else tt
    if null_data:
        return lib.agd_blend(n_patches, None, None, None, None, None, None, mode, taper, 1,
                             None, None, None, None, None, None)
    rc, _ = capi.call_blend(lib.agd_blend, np.float32, [5] if n_patches else [], st if n_patches else [],
                            ch, tt, data, mode, taper, [5], st, ch, tto)
    return rc


def test_blend_rejects(capfd):
    assert _blend(n_patches=0) == 1
    assert "n_patches must be > 0" in capfd.readouterr().err
    assert _blend(null_data=True) == 1
    assert "must not be NULL" in capfd.readouterr().err
    assert _blend(out_types=[np.array([0, 1, 0, 0], np.int32)]) == 1
    assert "Output trace types may not be AGDBad" in capfd.readouterr().err
    assert _blend(taper=-1, mode=A.AGDBlendMean) == 1
    assert "taper_length must be >= 0" in capfd.readouterr().err


def test_python_wrapper_errors(sv):
    """The Python layer raises like the reference wrapper
    (wrappers/python/agdeblend/agdeblend.py:78-100)."""
    with pytest.raises(RuntimeError, match="both must not be"):
        A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                  sv.trace_types, 1.0, 5, 0, sv.data, wavelet_idxs=[np.zeros(32, np.int32)])
    with pytest.raises(RuntimeError, match="same length as data"):
        A.deblend([0, 0], sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                  sv.trace_types, 1.0, 5, 0, sv.data)
    with pytest.raises(RuntimeError, match="Invalid blend_mode"):
        A.blend(sv.shottimes, sv.channels, sv.trace_types, sv.data, 7)
    with pytest.raises(RuntimeError, match="MPI"):
        A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                  sv.trace_types, 1.0, 5, 0, sv.data, comm=object())
