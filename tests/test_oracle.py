"""The oracle is pinned before it is trusted (CPU only):

* against the golden fixtures written by the reference's own operators
  (tests/golden/, made by tests/golden/make_golden.py);
* against the reference built here from its unchanged sources
  (oracle/_ref/, oracle/Makefile), when that build is present;
* the reference's own GoogleTest suite, compiled against the project-written
  FFTW3 and GoogleTest stand-ins, passes (when built).
"""
import os
import subprocess

import numpy as np
import pytest

import agd_oracle as O
import ref_bind
from agdeblend_b200 import synthetic as S
from agdeblend_b200.capi import DeblendArgs
from conftest import ROOT, rel_l2
from golden_io import GOLDEN, OPS_CASES, load_ops
from problems import random_problem

needs_ref = pytest.mark.skipif(not ref_bind.available(), reason="oracle/_ref not built")


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _interleave(x):
    return np.stack([x.real, x.imag], -1).reshape(-1)


@pytest.mark.parametrize("name", OPS_CASES)
def test_oracle_matches_golden(name):
    sv, ref = load_ops(name)
    plan = _plan(sv)
    assert abs(plan.step - ref["stepsize"]) <= 1e-15
    x = _interleave(O.model_to_flat(O.adjoint(plan, ref["record_in"])))
    assert rel_l2(x, ref["model_adjoint"]) <= 1e-12
    m = ref["model_adjoint"]
    y = O.forward(plan, O.flat_to_model(plan, m[0::2] + 1j * m[1::2]))
    assert rel_l2(y, ref["record_forward"]) <= 1e-12
    assert rel_l2(O.blend_input(plan, sv.data), ref["blend_input"]) == 0.0
    outs = O.set_output(plan, O.flat_to_model(plan, m[0::2] + 1j * m[1::2]))
    for o, r in zip(outs, ref["output"]):
        assert rel_l2(o, r) <= 1e-12


def test_golden_deblend_input_unchanged():
    """The synthetic gather the golden deblend output was made from is still
    generated identically."""
    g = np.load(os.path.join(GOLDEN, "gather_2d_deblend.npz"))
    sv = S.gather_2d()
    assert float(np.sum(sv.data[0].astype(np.float64))) == float(g["input_checksum"])
    # the reference output deblends the gather (sanity of the fixture)
    assert float(g["reference_snr_db"]) > 10.0


@needs_ref
@pytest.mark.parametrize("seed,kw", [(100, {}), (101, {}), (202, {"wavelets": True}),
                                     (301, {"neighbours": True}), (400, {"wavelets": True})])
def test_oracle_matches_reference_build(seed, kw):
    sv = random_problem(seed, **kw)
    args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.data, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets, dtype=np.float64)
    ref = ref_bind.RefOps(args)
    plan = _plan(sv)
    rec = np.random.default_rng(seed).standard_normal(ref.record_size)
    xr = ref.adjoint(rec)
    assert rel_l2(_interleave(O.model_to_flat(O.adjoint(plan, rec))), xr) <= 1e-12
    yo = O.forward(plan, O.flat_to_model(plan, xr[0::2] + 1j * xr[1::2]))
    assert rel_l2(yo, ref.forward(xr)) <= 1e-12
    assert abs(ref.stepsize - plan.step) <= 1e-15


@needs_ref
def test_oracle_deblend_matches_reference_double():
    """The full solver: oracle (float64, double schedule) vs the reference's
    double-precision agd_deblend."""
    sv = S.gather_2d(seed=31, n_shots=48, nt=256, window=(16, 128))
    args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.data, dtype=np.float64)
    assert ref_bind.ref_deblend(args, 1.0, 30) == 0
    out = O.deblend(_plan(sv), sv.data, 1.0, 30, double_schedule=True)
    assert rel_l2(out[0], args.data[0]) <= 1e-9


@needs_ref
def test_oracle_blend_matches_reference():
    sv = random_problem(705)
    nts = [d.shape[-1] for d in sv.data]
    flat = [d.reshape(-1, n) for d, n in zip(sv.data, nts)]
    for mode in (0, 1, 2):
        rc, res = ref_bind.ref_blend(np.float64, nts, sv.shottimes, sv.channels,
                                     sv.trace_types, flat, mode, 3, nts, sv.shottimes,
                                     sv.channels, [np.where(t == 1, 0, t) for t in sv.trace_types])
        assert rc == 0
        ref = O.blend(nts, sv.shottimes, sv.channels, sv.trace_types, flat, mode, 3, nts,
                      sv.shottimes, sv.channels, [np.where(t == 1, 0, t) for t in sv.trace_types])
        for a, b in zip(res, ref):
            assert rel_l2(a, b) <= 1e-14


def test_lambda_schedule_known_values():
    """first_linear_it truncation and decay for the benchmark iteration counts
    (src/agdeblend.c:526-533) evaluated in float and double."""
    for n_its in (100, 150, 200, 800):
        d, fli, slope = O.lambda_schedule(1.0, n_its)
        dd, fli_d, slope_d = O.lambda_schedule(1.0, n_its, double=True)
        assert abs(d - dd) <= 1e-6 and fli == fli_d
        assert 0 < fli < n_its
        lams = O.lambdas(1.0, 1.0, n_its)
        assert lams[-1] == 0.0 and abs(lams[0] - 1.0) < 1e-12


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_unit_tests")),
                    reason="reference unit tests not built")
def test_reference_unit_tests_pass_on_shim():
    """The reference's own GoogleTest suite (src/test.cpp and the *_test.cpp it
    includes) on the project FFTW3 stand-in; the 800-iteration end-to-end case
    is left to the GPU suite to keep this run short."""
    env = dict(os.environ, MINI_GTEST_SKIP="AGDeblend.Deblend")
    r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_unit_tests")],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "0 failed" in r.stdout


def test_sketch_estimates_relative_difference():
    """The sketch used by the full-size parity test: linear, and its relative
    difference tracks the true relative L2 difference."""
    from golden_io import sketch

    rng = np.random.default_rng(77)
    a = [rng.standard_normal((300, 700)), rng.standard_normal(5000)]
    e = [1e-3 * rng.standard_normal(x.shape) for x in a]
    b = [x + y for x, y in zip(a, e)]
    sa, sb, se = sketch(a), sketch(b), sketch(e)
    np.testing.assert_allclose(sb - sa, se, atol=1e-9)
    true = np.sqrt(sum(np.sum(y ** 2) for y in e) / sum(np.sum(x ** 2) for x in a))
    est = np.linalg.norm(sb - sa) / np.linalg.norm(sa)
    assert 0.5 * true < est < 2.0 * true
