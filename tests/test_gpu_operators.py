"""GPU parity of the operator A = mute . blend . wavelet . FK and its pieces
against the float64 oracle, through the C-ABI (include/agdeblend_gpu.h).

Tolerances: 1e-5 relative L2 in float (the stated operator gate), 1e-11 in
double; the dot-product test |<Ax, r> - <x, A^H r>| / |<Ax, r>| <= 1e-5
(float) / 1e-11 (double), as the reference's FK.DotTest and Model.DotTest
check the same identity (src/fk_test.cpp:547-660, src/model_test.cpp:598-835).
"""
import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from conftest import rel_l2
from problems import random_problem

pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-5, np.float64: 1e-11}


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _interleave(x):
    return np.stack([x.real, x.imag], -1).reshape(-1)


def _check_operators(sv, dtype, seed=0):
    tol = TOL[dtype]
    prob = A.Problem.from_survey(sv, dtype)
    plan = _plan(sv)
    assert prob.n_windows == len(plan.windows)
    assert prob.model_size == sum(plan.model_sizes)
    assert prob.record_size == plan.cfg.total
    assert abs(prob.stepsize - plan.step) <= 1e-6 * plan.step
    rng = np.random.default_rng(seed)
    rec = rng.standard_normal(prob.record_size)
    # the adjoint takes a residual, which is zero on muted samples; the
    # reference's dot test mutes its random record the same way
    # (src/model_test.cpp:790)
    O.apply_mute(plan.cfg, rec)
    # adjoint
    x_gpu = prob.adjoint(rec)
    x_ref = _interleave(O.model_to_flat(O.adjoint(plan, rec)))
    assert rel_l2(x_gpu, x_ref) <= tol, "adjoint"
    # forward of a Hermitian-consistent model (the adjoint of a record)
    y_gpu = prob.forward(x_ref)
    y_ref = O.forward(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    assert rel_l2(y_gpu, y_ref) <= tol, "forward"
    # dot test on GPU results alone
    lhs = float(np.dot(y_gpu.astype(np.float64), rec))
    rhs = float(np.dot(x_gpu.astype(np.float64), x_ref))
    assert abs(lhs - rhs) <= tol * max(abs(lhs), 1e-30), "dot test"
    # set_output and blend_input
    outs = prob.set_output(x_ref)
    outs_ref = O.set_output(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    for o, r in zip(outs, outs_ref):
        assert rel_l2(o, r) <= tol, "set_output"
    d_gpu = prob.blend_input(sv.data)
    d_ref = O.blend_input(plan, sv.data)
    d_tol = 1e-6 if dtype == np.float32 else 1e-12
    assert rel_l2(d_gpu, d_ref) <= d_tol, "blend_input"
    prob.close()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["gather_2d", "two_volume_3d", "vibroseis_4d"])
def test_operators_vs_oracle(small_surveys, name, dtype):
    _check_operators(small_surveys[name], dtype)


@pytest.mark.parametrize("seed", range(6))
def test_operators_random_problems(seed):
    _check_operators(random_problem(100 + seed), np.float32, seed)


@pytest.mark.parametrize("seed", range(3))
def test_operators_random_wavelets(seed):
    _check_operators(random_problem(200 + seed, wavelets=True), np.float32, seed)


@pytest.mark.parametrize("seed", range(3))
def test_operators_neighbour_patches(seed):
    _check_operators(random_problem(300 + seed, neighbours=True), np.float32, seed)


def test_operators_double_random():
    _check_operators(random_problem(400, wavelets=True), np.float64, 1)
