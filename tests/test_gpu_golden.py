"""GPU operators against the reference's own outputs recorded in
tests/golden/ (double-precision reference operators): 1e-5 relative L2 for
the float library, 1e-11 for the double library."""
import numpy as np
import pytest

import agdeblend_b200 as A
from conftest import rel_l2
from golden_io import OPS_CASES, load_ops

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("name", OPS_CASES)
def test_gpu_matches_reference_golden(name, dtype):
    tol = 1e-5 if dtype == np.float32 else 1e-11
    sv, ref = load_ops(name)
    prob = A.Problem.from_survey(sv, dtype)
    assert abs(prob.stepsize - ref["stepsize"]) <= (1e-6 if dtype == np.float32 else 1e-15)
    assert rel_l2(prob.adjoint(ref["record_in"]), ref["model_adjoint"]) <= tol
    assert rel_l2(prob.forward(ref["model_adjoint"]), ref["record_forward"]) <= tol
    assert rel_l2(prob.blend_input(sv.data), ref["blend_input"]) <= (1e-6 if dtype == np.float32
                                                                     else 1e-14)
    for o, r in zip(prob.set_output(ref["model_adjoint"]), ref["output"]):
        assert rel_l2(o, r) <= tol
    prob.close()
