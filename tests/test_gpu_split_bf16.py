"""The split-BF16 tensor-core space kernels (precision mode 1,
agd_gpu_problem_set_precision) against the float64 operator oracle.

The space DFTs of windows (16, 16, 16, nt) become hi + lo BF16 products with
FP32 accumulation (about 16 significant bits per operand) on tcgen05; the
time axis stays FP32.  Stated error bounds (relative L2 against the FP64
oracle): forward and adjoint 1e-4 (the FP32 kernels: 1e-5), dot test 1e-4;
a solve stays within 1e-3 of the FP32 solve, SNR within 0.05 dB."""
import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_OP = 1e-4


def _survey(seed=41, wavelet=True, nt=300):
    """2 x 2 windows of 16^3 over a (24, 24, 16, nt) volume (padded space
    shape 20^3), time window 64; a 40-sample sweep wavelet or none."""
    sv = S.vibroseis_4d(seed=seed, n_sy=24, n_sx=24, n_ch=16, nt=nt,
                        window=(16, 16, 16, 64), wavelet_len=40, n_its=30)
    if not wavelet:
        sv.wavelet_lengths = sv.wavelet_idxs = sv.wavelets = None
    return sv


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _interleave(x):
    return np.stack([x.real, x.imag], -1).reshape(-1)


@pytest.mark.parametrize("wavelet", [False, True])
def test_split_bf16_operators_vs_fp64_oracle(wavelet):
    sv = _survey(wavelet=wavelet)
    prob = A.Problem.from_survey(sv)
    n_tc = prob.set_precision(A.Problem.PRECISION_SPLIT_BF16)
    assert n_tc == prob.n_windows == 4
    assert prob.kernels()["space_fwd"] == "space_fwd_tc"
    plan = _plan(sv)
    rng = np.random.default_rng(5)
    rec = rng.standard_normal(prob.record_size)
    O.apply_mute(plan.cfg, rec)
    x_gpu = prob.adjoint(rec)
    x_ref = _interleave(O.model_to_flat(O.adjoint(plan, rec)))
    err_adj = rel_l2(x_gpu, x_ref)
    y_gpu = prob.forward(x_ref)
    y_ref = O.forward(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    err_fwd = rel_l2(y_gpu, y_ref)
    lhs = float(np.dot(y_gpu.astype(np.float64), rec))
    rhs = float(np.dot(x_gpu.astype(np.float64), x_ref))
    err_dot = abs(lhs - rhs) / abs(lhs)
    print(f"split-BF16 relative L2 vs FP64 oracle: adjoint {err_adj:.2e} forward "
          f"{err_fwd:.2e} dot {err_dot:.2e}")
    assert err_adj <= TOL_OP and err_fwd <= TOL_OP and err_dot <= TOL_OP
    # not the FP32 kernels in disguise: their error is two orders smaller
    prob.set_precision(A.Problem.PRECISION_FP32)
    assert rel_l2(prob.adjoint(rec), x_ref) < 0.1 * err_adj
    prob.close()


def test_split_bf16_solve_matches_fp32_solve():
    sv = _survey(seed=42)
    prob = A.Problem.from_survey(sv)
    ref = prob.solve(sv.data, 1.0, 30)
    assert prob.set_precision(A.Problem.PRECISION_SPLIT_BF16) == 4
    out = prob.solve(sv.data, 1.0, 30)
    prob.close()
    for o, r in zip(out, ref):
        assert np.isfinite(o).all()
        assert rel_l2(o, r) <= 1e-3
    assert abs(S.snr_db(out, sv.truth, sv.trace_types) -
               S.snr_db(ref, sv.truth, sv.trace_types)) <= 0.05


def test_split_bf16_rejected_by_double_library():
    sv = _survey(seed=43, wavelet=False)
    prob = A.Problem.from_survey(sv, np.float64)
    with pytest.raises(RuntimeError):
        prob.set_precision(A.Problem.PRECISION_SPLIT_BF16)
    prob.close()
