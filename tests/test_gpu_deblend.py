"""End-to-end GPU parity of agd_deblend / agd_blend through the public C API.

Gates: the deblended output after the same n_its is within 1e-3 relative L2
of the float64 oracle (and of the reference's own float output where it was
recorded), and its SNR against the unblended truth matches to 0.05 dB.  The
reference-style quality test repeats src/test.cpp:432-561 (five random
problems, 800 iterations, error energy below a tenth of the signal energy).
"""
import os

import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import ROOT, rel_l2
from problems import random_problem
from residual_cases import CASES as RESIDUAL_CASES
from residual_cases import make_case as residual_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _deblend(sv, n_its=None):
    return A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                     sv.trace_types, sv.initial_factor, n_its or sv.n_its, 0, sv.data,
                     wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)


def test_gather_2d_full_vs_oracle():
    """The 128-shot x 512-sample gather, window (32, 256), 100 iterations."""
    sv = S.gather_2d()
    out = _deblend(sv)
    ref = O.deblend(_plan(sv), sv.data, sv.initial_factor, sv.n_its)
    assert rel_l2(out[0], ref[0]) <= 1e-3
    snr_gpu = S.snr_db(out, sv.truth, sv.trace_types)
    snr_ref = S.snr_db(ref, sv.truth, sv.trace_types)
    assert abs(snr_gpu - snr_ref) <= 0.05
    path = os.path.join(GOLDEN, "gather_2d_deblend.npz")
    if os.path.exists(path):
        g = np.load(path)
        assert rel_l2(out[0], g["reference_out"]) <= 1e-3
        assert abs(snr_gpu - float(g["reference_snr_db"])) <= 0.05


@pytest.mark.parametrize("name", ["two_volume_3d", "vibroseis_4d"])
def test_small_surveys_vs_oracle(small_surveys, name):
    sv = small_surveys[name]
    out = _deblend(sv)
    ref = O.deblend(_plan(sv), sv.data, sv.initial_factor, sv.n_its)
    for o, r in zip(out, ref):
        assert rel_l2(o, r) <= 1e-3
    assert abs(S.snr_db(out, sv.truth, sv.trace_types) -
               S.snr_db(ref, sv.truth, sv.trace_types)) <= 0.05


@pytest.mark.parametrize("seed,kw", [(800, {}), (801, {}), (802, {"wavelets": True}),
                                     (803, {"neighbours": True}), (804, {"neighbours": True})])
def test_solve_random_problems(seed, kw):
    sv = random_problem(seed, **kw)
    prob = A.Problem.from_survey(sv)
    out = prob.solve(sv.data, 1.0, 25)
    ref = O.deblend(_plan(sv), sv.data, 1.0, 25)
    for o, r in zip(out, ref):
        assert rel_l2(o, r) <= 1e-3
    prob.close()


def test_repeated_solves_and_print_path_agree():
    """Solves replay one captured CUDA graph per problem; a second solve on
    the same problem (graph reused, longer schedule) and the printing path
    (launched without the graph) must give the same output."""
    sv = S.gather_2d(seed=9, n_shots=48, nt=256, window=(16, 128))
    prob = A.Problem.from_survey(sv)
    a = prob.solve(sv.data, 1.0, 15)
    b = prob.solve(sv.data, 1.0, 15)
    c = prob.solve(sv.data, 1.0, 40)
    d = prob.solve(sv.data, 1.0, 40, print_freq=7)
    ref = O.deblend(_plan(sv), sv.data, 1.0, 40)
    assert np.array_equal(a[0], b[0])
    assert rel_l2(c[0], d[0]) <= 1e-6
    assert rel_l2(c[0], ref[0]) <= 1e-3
    prob.close()


def test_double_library_vs_oracle(small_surveys):
    sv = small_surveys["two_volume_3d"]
    data64 = [d.astype(np.float64) for d in sv.data]
    out = A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                    sv.trace_types, sv.initial_factor, sv.n_its, 0, data64)
    ref = O.deblend(_plan(sv), sv.data, sv.initial_factor, sv.n_its, double_schedule=True)
    for o, r in zip(out, ref):
        assert o.dtype == np.float64
        assert rel_l2(o, r) <= 1e-8


def test_reference_quality_random_problems():
    """src/test.cpp:432-561: blend random problems, deblend 800 iterations."""
    for k in range(5):
        sv = random_problem(500 + k, bad_missing=False, max_dims=4)
        rng = np.random.default_rng(600 + k)
        truth = []
        for d in sv.data:
            nt = d.shape[-1]
            tv = (rng.uniform(size=nt) - 0.5).astype(np.float32)
            truth.append(np.broadcast_to(tv, d.shape).copy())
        nts = [d.shape[-1] for d in truth]
        blended = A.blend(sv.shottimes, sv.channels, sv.trace_types,
                          [t.reshape(-1, n) for t, n in zip(truth, nts)], A.AGDBlendSum)
        data = [b.reshape(t.shape) for b, t in zip(blended, truth)]
        out = A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                        sv.trace_types, 1.0, 800, 0, data)
        err = sum(float(np.sum((o - t) ** 2)) for o, t in zip(out, truth))
        tru = sum(float(np.sum(t ** 2)) for t in truth)
        assert err < tru / 10


@pytest.mark.parametrize("mode", [A.AGDBlendSum, A.AGDBlendMean, A.AGDBlendOverwrite])
@pytest.mark.parametrize("taper", [0, 5])
def test_blend_vs_oracle(mode, taper):
    sv = random_problem(700 + mode, bad_missing=True)
    nts = [d.shape[-1] for d in sv.data]
    flat = [d.reshape(-1, n) for d, n in zip(sv.data, nts)]
    rng = np.random.default_rng(mode)
    st_out = [s + rng.integers(-3, 4, s.shape) for s in sv.shottimes]
    tt_out = [np.where(t == 1, 0, t).astype(np.int32) for t in sv.trace_types]
    nt_out = [n + 2 for n in nts]
    out = A.blend(sv.shottimes, sv.channels, sv.trace_types, flat, mode, taper_length=taper,
                  n_times_out=nt_out, shottimes_out=st_out, channels_out=sv.channels,
                  trace_types_out=tt_out)
    ref = O.blend(nts, sv.shottimes, sv.channels, sv.trace_types, flat, mode, taper, nt_out,
                  st_out, sv.channels, tt_out)
    for o, r in zip(out, ref):
        assert rel_l2(o.reshape(r.shape), r) <= 1e-6


def test_print_freq_lines(capfd):
    sv = S.gather_2d(seed=5, n_shots=32, nt=256, window=(16, 128))
    A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
              sv.trace_types, 1.0, 6, 2, sv.data)
    out = capfd.readouterr().out
    lines = [ln for ln in out.splitlines() if ln.startswith("Iteration")]
    assert [ln.split()[1] for ln in lines] == ["0", "2", "4"]


def _residual_lines(text):
    its, vals = [], []
    for ln in text.splitlines():
        parts = ln.split()
        if len(parts) == 4 and parts[0] == "Iteration" and parts[2] == "Residual":
            its.append(int(parts[1]))
            vals.append(float(parts[3]))
    return np.array(its), np.array(vals)


@pytest.mark.parametrize("name", RESIDUAL_CASES)
def test_print_freq_residuals_match_reference(name, capfd):
    """The residual norms printed with print_freq > 0 (FP64 on the device)
    against the lines the reference float build printed on the same survey
    (tests/golden/make_residual_fixture.py): same iterations, values within
    1e-3 relative."""
    ref = np.load(os.path.join(GOLDEN, "residual_lines_reference.npz"))
    sv, print_freq = residual_case(name)
    kw = {}
    if sv.wavelets is not None:
        kw = dict(wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)
    capfd.readouterr()
    A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
              sv.trace_types, sv.initial_factor, sv.n_its, print_freq, sv.data, **kw)
    its, vals = _residual_lines(capfd.readouterr().out)
    assert np.array_equal(its, ref[f"{name}_its"])
    want = ref[f"{name}_residual"]
    assert np.all(np.abs(vals - want) <= 1e-3 * np.abs(want) + 1e-6)


def test_overwrite_input_writes_the_result_in_place():
    """deblend(..., overwrite_input=True) returns the caller's own arrays,
    holding the same result as the default call (which leaves them intact)."""
    sv = S.gather_2d(seed=77, n_its=20)
    out = _deblend(sv, 20)
    before = [d.copy() for d in sv.data]
    assert all(np.array_equal(a, b) for a, b in zip(sv.data, before))
    buf = [d.copy() for d in sv.data]
    res = A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                    sv.trace_types, sv.initial_factor, 20, 0, buf, overwrite_input=True)
    assert np.shares_memory(res[0], buf[0])
    assert np.array_equal(res[0], out[0])
