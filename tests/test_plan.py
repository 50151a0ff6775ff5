"""The C++ host planning (agdeblend_b200/csrc/plan.cpp) against the oracle's
restatement of set_model / set_blend_config, through agd_plan_export (no GPU
is touched): window geometry, FK constants, record layout, mute spans and
every window trace's blend coordinates."""
import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from golden_io import OPS_CASES, load_ops
from problems import random_problem


def _compare(sv):
    info, win, bl = A.plan_export(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords,
                                  sv.shapes, sv.shottimes, sv.channels, sv.trace_types,
                                  sv.wavelet_lengths, sv.wavelet_idxs, sv.wavelets)
    plan = O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)
    assert info[0] == len(plan.windows)
    assert info[1] == sum(plan.model_sizes)
    assert info[2] == plan.cfg.total
    assert info[4] == sum(len(c) for c in plan.cfg.intervals)
    assert info[5] == len(plan.cfg.mute)
    for w, row in zip(plan.windows, win):
        D = len(w.shape)
        assert row[0] == w.patch and row[1] == D
        assert list(row[2:10]) == [w.n_tw, w.n_freq, w.lt, w.padded[-1], w.lt // 2, w.n_fk,
                                   w.conv, w.n_traces]
        assert list(row[10:10 + D]) == list(w.shape)
        assert list(row[14:14 + D]) == list(w.padded[:-1])
        assert list(row[18:18 + 2 * D]) == list(w.use_taper)
    expect = np.array([c if c is not None else (-1, 0, 0)
                       for w in plan.windows for c in w.blend], np.int64).reshape(-1, 3)
    got = bl.copy()
    got[got[:, 0] < 0] = (-1, 0, 0)
    assert np.array_equal(got, expect)


@pytest.mark.parametrize("seed", range(20))
def test_plan_random_problems(seed):
    _compare(random_problem(1000 + seed, wavelets=seed % 3 == 0, neighbours=seed % 4 == 1))


@pytest.mark.parametrize("name", OPS_CASES)
def test_plan_golden_cases(name):
    _compare(load_ops(name)[0])


def test_plan_benchmark_survey():
    """The benchmark survey: 98 windows, 113.6 M complex model values, and
    exactly three record intervals per channel (the two gaps)."""
    sv = S.two_volume_3d()
    info, win, bl = A.plan_export(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords,
                                  sv.shapes, sv.shottimes, sv.channels, sv.trace_types)
    assert info[0] == 98
    assert info[1] == 98 * 9 * 161 * 20 * 40
    assert info[4] == 64 * 3
    assert (win[:, 2] == 9).all() and (win[:, 5] == 320).all()


def test_plan_gather_sizes():
    """The 2-D gather: 7 windows of padded shape (40, 320), 5 time windows,
    n_times_fk = n_times_conv = 768, 225,400 complex model values."""
    sv = S.gather_2d()
    info, win, bl = A.plan_export(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords,
                                  sv.shapes, sv.shottimes, sv.channels, sv.trace_types)
    assert info[0] == 7 and info[1] == 225400
    assert (win[:, 2] == 5).all() and (win[:, 7] == 768).all() and (win[:, 8] == 768).all()
    assert (win[:, 14] == 40).all() and (win[:, 5] == 320).all()


def test_plan_enlarged_windows():
    """Uneven split of 78 traces into nominal 32-wide windows gives lengths
    37, 37, 36 (src/model_test.cpp:272-326)."""
    rng = np.random.default_rng(3)
    n = 78
    sv = S.Survey("uneven", [0], [2], [[32, 64]], [[0]], [[n, 100]],
                  [np.arange(n, dtype=np.int64) * 40], [np.zeros(n, np.int32)],
                  [np.zeros(n, np.int32)], [rng.standard_normal((n, 100)).astype(np.float32)],
                  [None], 5)
    info, win, bl = A.plan_export(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords,
                                  sv.shapes, sv.shottimes, sv.channels, sv.trace_types)
    assert list(win[:, 10]) == [37, 37, 36]
    _compare(sv)
