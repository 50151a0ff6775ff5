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


def _merge_survey(seed, n_traces=400, nt=16):
    """One 2-D patch whose trace spans overlap, touch and arrive out of
    order on three channels: shot times on a grid of half a trace, so that
    new spans often touch several list entries at once (the cases where the
    reference's merge scan skips an entry)."""
    rng = np.random.default_rng(seed)
    st = (rng.integers(0, 60, n_traces) * (nt // 2)).astype(np.int64)
    ch = rng.integers(0, 3, n_traces).astype(np.int32)
    tt = rng.choice([S.LIVE, S.LIVE, S.LIVE, S.BAD, S.MISSING], n_traces).astype(np.int32)
    tt[0] = S.LIVE
    data = np.zeros((n_traces, nt), np.float32)
    return S.Survey("merge", [0], [2], [[n_traces, nt]], [[0]], [[n_traces, nt]], [st], [ch],
                    [tt], [data], [data], 1)


@pytest.mark.parametrize("seed", range(12))
def test_interval_merge_order_matches_reference(seed):
    """The sort-based merge (plan.cpp IntervalList) against the oracle's
    list scan, record layout, mute spans and blend coordinates included."""
    _compare(_merge_survey(500 + seed))


def test_planning_scales_to_a_million_traces():
    """256 channels x 4096 shots x 64 samples with records that never touch:
    4096 record intervals per channel (an interval search per trace would
    scan 8 M entries per channel)."""
    import time

    n_ch, n_shots, nt = 256, 4096, 64
    # record spans are C = 128 samples long (the padded time length of the
    # 64-sample windows): shots 200 samples apart never touch
    st = np.repeat((np.arange(n_shots) * 200).astype(np.int64)[None, :], n_ch, 0)
    ch = np.repeat(np.arange(n_ch, dtype=np.int32)[:, None], n_shots, 1)
    tt = np.zeros((n_ch, n_shots), np.int32)
    t0 = time.perf_counter()
    info, win, bl = A.plan_export([0], [3], [[16, 32, 64]], [[0, 0]], [[n_ch, n_shots, nt]],
                                  [st], [ch], [tt])
    dt = time.perf_counter() - t0
    conv = int(win[0, 8])
    assert conv == 128
    assert info[4] == n_ch * n_shots  # one record interval per trace
    assert info[2] == n_ch * n_shots * conv
    assert dt < 30.0
