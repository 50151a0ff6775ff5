"""GPU parity of the line-DFT space kernels (line_dft.cuh): windows with one
space axis whose padded length P has no shape-specialised kernel (enlarged
edge windows such as L = 33 -> P = 42, prime P = 43, 83, 89, 127, every P
up to 128), against the float64 oracle through the C-ABI.

Each case first checks that the line kernels serve the windows (info[22]),
so that a silent fallback to the generic FFT passes cannot pass the test;
the operator checks are those of test_gpu_operators (1e-5 relative L2 and
the dot test in float, 1e-11 in double).  Solves are compared with the
generic FFT passes (AGD_GPU_GENERIC=1), and a batch of gathers on the line
kernels with the same gathers solved one by one."""
import dataclasses
import os

import numpy as np
import pytest

import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import rel_l2
from test_gpu_operators import _check_operators

pytestmark = pytest.mark.gpu

# (shots per window, shots in the gather) -> padded lengths of its windows
CASES = {
    "P42_even_enlarged": (32, 67),
    "P43_prime": (32, 88),
    "P83_prime": (64, 165),
    "P84_even": (64, 67),
    "P88_P89": (64, 109),
    "P125_P127": (100, 151),
    "P128_largest": (100, 102),
    "P22_short": (16, 60),
}


def _gather(name, seed=4100):
    ws, n = CASES[name]
    return S.gather_2d(seed=seed, n_shots=n, nt=300, window=(ws, 128))


def _line_windows(sv, dtype=np.float32):
    prob = A.Problem.from_survey(sv, dtype)
    n_line, n_win = int(prob.info[22]), prob.n_windows
    prob.close()
    return n_line, n_win


@pytest.mark.parametrize("name", sorted(CASES))
def test_line_operators_vs_oracle(name):
    sv = _gather(name)
    n_line, _ = _line_windows(sv)
    assert n_line > 0, "no window on the line kernels"
    _check_operators(sv, np.float32)


@pytest.mark.parametrize("name", ["P83_prime", "P128_largest", "P42_even_enlarged"])
def test_line_operators_double(name):
    sv = _gather(name, seed=4200)
    assert _line_windows(sv, np.float64)[0] > 0
    _check_operators(sv, np.float64, 1)


@pytest.mark.parametrize("name", ["P83_prime", "P42_even_enlarged"])
def test_line_operators_with_wavelet(name):
    # a source wavelet on every live trace: the wavelet stage runs on the
    # traces around the line kernels' space transforms
    sv = _gather(name, seed=4600)
    rng = np.random.default_rng(4601)
    w = (rng.standard_normal(24) * np.hanning(24)).astype(np.float32)
    n_tr = int(np.asarray(sv.trace_types[0]).size)
    sv = dataclasses.replace(sv, wavelet_lengths=[len(w)],
                             wavelet_idxs=[np.zeros(n_tr, np.int32)], wavelets=[w])
    assert _line_windows(sv)[0] > 0
    _check_operators(sv, np.float32)


def test_lengths_above_the_limit_stay_generic():
    # shots 207 with 100-shot windows give P = 129 windows beside shorter ones
    sv = S.gather_2d(seed=4300, n_shots=207, nt=300, window=(100, 128))
    info, win, _ = A.plan_export(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords,
                                 sv.shapes, sv.shottimes, sv.channels, sv.trace_types)
    P = win[:, 14]
    n_line, n_win = _line_windows(sv)
    assert n_line == int(np.sum((P <= 128) & (P != 20) & (P != 40)))
    assert n_line < n_win
    _check_operators(sv, np.float32)


def _solve(sv, n_its, generic):
    old = os.environ.get("AGD_GPU_GENERIC")
    if generic:
        os.environ["AGD_GPU_GENERIC"] = "1"
    try:
        return A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                         sv.trace_types, 1.0, n_its, 0, sv.data)
    finally:
        if old is None:
            os.environ.pop("AGD_GPU_GENERIC", None)
        else:
            os.environ["AGD_GPU_GENERIC"] = old


@pytest.mark.parametrize("name", ["P83_prime", "P84_even", "P125_P127"])
def test_line_solve_matches_generic_passes(name):
    sv = _gather(name, seed=4400)
    out = _solve(sv, 20, generic=False)
    ref = _solve(sv, 20, generic=True)
    for o, r in zip(out, ref):
        assert rel_l2(o, r) <= 1e-4


def test_line_batch_matches_separate_solves():
    gathers = [_gather(n, seed=4500 + i) for i, n in
               enumerate(["P83_prime", "P42_even_enlarged", "P128_largest", "P22_short"])]
    kw = [dict(volumes=g.volumes, window_shapes=g.window_shapes, coords=g.coords,
               shottimes=g.shottimes, channels=g.channels, trace_types=g.trace_types,
               data=g.data) for g in gathers]
    outs = A.deblend_batch(kw, 1.0, 15)
    for g, out in zip(gathers, outs):
        ref = _solve(g, 15, generic=False)
        for o, r in zip(out, ref):
            assert rel_l2(o, r) <= 1e-5
