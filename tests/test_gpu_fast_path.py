"""The shape-specialised kernels (agdeblend_b200/csrc/fast.cuh) against the
oracle, for every instantiated window shape and every candidate of the
space-kernel autotuner (forced with AGD_GPU_SPACE_VARIANT), and against the
generic kernels (forced with AGD_GPU_GENERIC=1) on the same problem."""
import os

import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import rel_l2

pytestmark = pytest.mark.gpu

# (space shape, time samples, window) -> padded space lengths hit
CASES = [
    ("1d_P40", lambda: S.gather_2d(seed=41, n_shots=64, nt=300, window=(32, 128))),
    ("1d_P20", lambda: S.gather_2d(seed=42, n_shots=48, nt=600, window=(16, 256))),
    ("2d_P20x40", lambda: S.two_volume_3d(seed=43, n_ch=32, n_shots=64, nt=300,
                                          window=(16, 32, 128))),
    ("2d_P20x20", lambda: S.two_volume_3d(seed=44, n_ch=32, n_shots=32, nt=300,
                                          window=(16, 16, 128))),
    ("2d_P40x40", lambda: S.two_volume_3d(seed=45, n_ch=32, n_shots=64, nt=300,
                                          window=(32, 32, 256))),
    ("3d_P20x20x20", lambda: S.vibroseis_4d(seed=46, n_sy=16, n_sx=16, n_ch=16, nt=200,
                                            window=(16, 16, 16, 128), wavelet_len=1)),
]


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _interleave(x):
    return np.stack([x.real, x.imag], -1).reshape(-1)


def _problem(sv, generic=False, dtype=np.float32, variant=None, time_variant=None):
    env = {"AGD_GPU_GENERIC": "1" if generic else "0",
           "AGD_GPU_SPACE_VARIANT": "" if variant is None else f"{variant[0]},{variant[1]}",
           "AGD_GPU_TIME_VARIANT": "" if time_variant is None else
           f"{time_variant[0]},{time_variant[1]}"}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return A.Problem.from_survey(sv, dtype)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _check_operators(sv, prob, tol):
    plan = _plan(sv)
    rng = np.random.default_rng(1)
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
    assert abs(lhs - rhs) <= tol * abs(lhs)
    outs = prob.set_output(x_ref)
    ref_out = O.set_output(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    for o, r in zip(outs, ref_out):
        assert rel_l2(o, r) <= tol


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_fast_operators_vs_oracle(name, make, dtype):
    tol = 1e-5 if dtype == np.float32 else 1e-11
    sv = make()
    prob = _problem(sv, dtype=dtype)
    assert prob.info[8] == 1
    assert 0 <= prob.info[10] < prob.info[12] and 0 <= prob.info[11] < prob.info[13]
    _check_operators(sv, prob, tol)
    prob.close()


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_every_space_candidate_vs_oracle(name, make):
    """Each forward/adjoint candidate the set-up timing may pick."""
    sv = make()
    probe = _problem(sv)
    n_f, n_a = int(probe.info[12]), int(probe.info[13])
    probe.close()
    assert n_f >= 1 and n_a >= 1
    for v in range(max(n_f, n_a)):
        pick = (min(v, n_f - 1), min(v, n_a - 1))
        prob = _problem(sv, variant=pick)
        assert (prob.info[10], prob.info[11]) == pick
        _check_operators(sv, prob, 1e-5)
        prob.close()


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_every_time_candidate_vs_oracle(name, make):
    """Each time-kernel candidate (traces per block, line stride) the set-up
    timing may pick."""
    sv = make()
    probe = _problem(sv)
    n = int(probe.info[19])
    probe.close()
    assert n >= 1
    for v in range(n):
        prob = _problem(sv, time_variant=(v, v))
        assert (prob.info[17], prob.info[18]) == (v, v)
        _check_operators(sv, prob, 1e-5)
        prob.close()


@pytest.mark.parametrize("name,make", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_fast_solve_matches_generic_and_oracle(name, make):
    sv = make()
    fast = _problem(sv)
    generic = _problem(sv, generic=True)
    assert fast.info[8] == 1 and generic.info[8] == 0
    out_f = fast.solve(sv.data, 1.0, 20)
    out_g = generic.solve(sv.data, 1.0, 20)
    ref = O.deblend(_plan(sv), sv.data, 1.0, 20)
    for a, b, r in zip(out_f, out_g, ref):
        assert rel_l2(a, r) <= 1e-3
        assert rel_l2(a, b) <= 1e-3
    fast.close()
    generic.close()
