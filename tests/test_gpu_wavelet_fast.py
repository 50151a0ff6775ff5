"""The prime-factor wavelet kernel (agdeblend_b200/csrc/wavelet_fast.cuh)
against the oracle and against the generic wavelet kernel (forced with
AGD_GPU_GENERIC=1): trace lengths of one to three coprime factors, even and
odd, pairs of traces with different spectra (several wavelets, bad and
missing traces), odd trace counts, and the 4-D vibroseis trace length
2431 = 11 * 13 * 17."""
import os

import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import rel_l2
from problems import random_problem

pytestmark = pytest.mark.gpu

_FACTORS = {2, 3, 4, 5, 7, 8, 9, 11, 13, 16, 17, 19, 23, 25, 27, 32}


def prime_powers(n):
    out, p = [], 2
    while n > 1:
        if n % p == 0:
            q = 1
            while n % p == 0:
                n //= p
                q *= p
            out.append(q)
        p += 1
    return out


def pfa_supported(c):
    f = prime_powers(c)
    return len(f) <= 4 and all(x in _FACTORS for x in f)


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _interleave(x):
    return np.stack([x.real, x.imag], -1).reshape(-1)


def _problem(sv, dtype, generic=False):
    old = os.environ.get("AGD_GPU_GENERIC")
    os.environ["AGD_GPU_GENERIC"] = "1" if generic else "0"
    try:
        return A.Problem.from_survey(sv, dtype)
    finally:
        if old is None:
            del os.environ["AGD_GPU_GENERIC"]
        else:
            os.environ["AGD_GPU_GENERIC"] = old


def _vibroseis_small(seed=61):
    """4-D vibroseis geometry with the full 2048-sample traces and 256-sample
    sweep (trace length 2431), 8 x 8 x 8 traces, with bad and missing traces
    so that trace pairs mix spectra."""
    sv = S.vibroseis_4d(seed=seed, n_sy=8, n_sx=8, n_ch=8, nt=2048, window=(8, 8, 8, 256))
    rng = np.random.default_rng(seed)
    tt = sv.trace_types[0].copy()
    tt[rng.random(tt.size) < 0.1] = S.BAD
    tt[rng.random(tt.size) < 0.05] = S.MISSING
    tt[0] = S.LIVE
    sv.trace_types = [tt]
    return sv


def _unscale(out, sv, plan, p):
    """set_output gives traces without a spectrum (bad, missing) C times
    their window prediction (the bare transform pair of src/wavelet.c:273).
    A model made by the adjoint of a muted record predicts about zero there,
    so those traces hold float rounding times C; dividing them by C compares
    every trace on the scale of its prediction."""
    o = np.array(out, np.float64).reshape(-1, out.shape[-1])
    non_live = np.asarray(sv.trace_types[p]).reshape(-1) != S.LIVE
    o[non_live] /= plan.conv[p]
    return o


def _check(sv, dtype, seed):
    tol = 1e-5 if dtype == np.float32 else 1e-11
    plan = _plan(sv)
    cs = sorted({w.conv for w in plan.windows})
    expect = all(pfa_supported(c) for c in cs)
    prob = _problem(sv, dtype)
    assert prob.info[9] == (1 if expect else 0), cs
    rng = np.random.default_rng(seed)
    rec = rng.standard_normal(prob.record_size)
    O.apply_mute(plan.cfg, rec)
    x_gpu = prob.adjoint(rec)
    x_ref = _interleave(O.model_to_flat(O.adjoint(plan, rec)))
    assert rel_l2(x_gpu, x_ref) <= tol
    y_gpu = prob.forward(x_ref)
    y_ref = O.forward(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    assert rel_l2(y_gpu, y_ref) <= tol
    lhs = float(np.dot(y_gpu.astype(np.float64), rec))
    rhs = float(np.dot(x_gpu.astype(np.float64), x_ref))
    assert abs(lhs - rhs) <= 10 * tol * abs(lhs)
    outs = prob.set_output(x_ref)
    ref_out = O.set_output(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    for p, (o, r) in enumerate(zip(outs, ref_out)):
        assert rel_l2(_unscale(o, sv, plan, p), _unscale(r, sv, plan, p)) <= tol
    if expect:
        gen = _problem(sv, dtype, generic=True)
        assert gen.info[9] == 0
        assert rel_l2(x_gpu, gen.adjoint(rec)) <= tol
        assert rel_l2(y_gpu, gen.forward(x_ref)) <= tol
        gen.close()
    prob.close()
    return expect


def test_pfa_rule_covers_the_test_lengths():
    assert prime_powers(2431) == [11, 13, 17] and pfa_supported(2431)
    assert pfa_supported(30) and pfa_supported(16) and not pfa_supported(31)
    assert not pfa_supported(64) and not pfa_supported(2 * 3 * 5 * 7 * 11)


# seeds chosen for their trace lengths: 0 (16, 20, 21; odd trace counts),
# 3 (31: generic kernel), 8 (30 = 2 * 3 * 5), 13 (16, 24, 32), 18 (22, 25, 35),
# 22 (16, 17, 25), 36 (24, 34)
@pytest.mark.parametrize("seed", [0, 3, 8, 13, 18, 22, 36])
def test_wavelet_fast_random_problems(seed):
    _check(random_problem(seed, wavelets=True), np.float32, seed)


@pytest.mark.parametrize("seed", [8, 22])
def test_wavelet_fast_random_problems_double(seed):
    _check(random_problem(seed, wavelets=True), np.float64, seed)


def test_wavelet_fast_vibroseis_length_2431():
    sv = _vibroseis_small()
    assert _check(sv, np.float32, 5)


def test_every_wavelet_candidate_vs_oracle():
    """Each wavelet-kernel candidate (blocks per SM, pairs per block) the
    set-up timing may pick, on the 2431-sample traces."""
    sv = _vibroseis_small(63)
    probe = _problem(sv, np.float32)
    n = int(probe.info[21])
    probe.close()
    assert n >= 1
    old = os.environ.get("AGD_GPU_WAVELET_VARIANT")
    try:
        for v in range(n):
            os.environ["AGD_GPU_WAVELET_VARIANT"] = str(v)
            prob = _problem(sv, np.float32)
            assert prob.info[20] == v
            plan = _plan(sv)
            rec = np.random.default_rng(v).standard_normal(prob.record_size)
            O.apply_mute(plan.cfg, rec)
            x_ref = _interleave(O.model_to_flat(O.adjoint(plan, rec)))
            assert rel_l2(prob.adjoint(rec), x_ref) <= 1e-5
            y_ref = O.forward(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
            assert rel_l2(prob.forward(x_ref), y_ref) <= 1e-5
            prob.close()
    finally:
        if old is None:
            os.environ.pop("AGD_GPU_WAVELET_VARIANT", None)
        else:
            os.environ["AGD_GPU_WAVELET_VARIANT"] = old


def test_wavelet_fast_solve_matches_oracle():
    sv = _vibroseis_small(62)
    prob = _problem(sv, np.float32)
    assert prob.info[9] == 1
    out = prob.solve(sv.data, 1.0, 15)
    ref = O.deblend(_plan(sv), sv.data, 1.0, 15)
    for a, r in zip(out, ref):
        assert rel_l2(a, r) <= 1e-3
    prob.close()
