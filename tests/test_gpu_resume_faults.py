"""Checkpoint / resume of the solver (agd_gpu_solve_range) and the error
paths of device allocation (the AGD_GPU_FAIL_ALLOC test hook).

Resume: the solver state is the model and the iteration number, so stopping
after iteration k and resuming from the returned model must reproduce the
uninterrupted solve.  Allocation failures: every device allocation of a call
is made to fail in turn; each call must return 1 (a RuntimeError in Python)
and give back all the device memory it took.  No failure here touches the
GPU itself: the hook only reports an error before the allocation."""
import os

import numpy as np
import pytest

import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import rel_l2
from problems import random_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: S.gather_2d(seed=3200, n_shots=96, nt=400),
                                  lambda: random_problem(8, wavelets=True)],
                         ids=["gather", "wavelets"])
def test_resume_reproduces_uninterrupted_solve(make):
    sv = make()
    prob = A.Problem.from_survey(sv)
    full = prob.solve(sv.data, 1.0, 20)
    part, model = prob.solve_range(sv.data, 1.0, 20, 0, 8)
    rest, _ = prob.solve_range(sv.data, 1.0, 20, 8, 20, model_in=model)
    for a, b in zip(rest, full):
        assert rel_l2(a, b) <= 1e-6
    # stopping at iteration 8 leaves the first part's model and its output
    again, model2 = prob.solve_range(sv.data, 1.0, 20, 0, 8)
    assert np.array_equal(model, model2)
    assert not all(rel_l2(a, b) <= 1e-6 for a, b in zip(part, full))
    prob.close()


def test_resume_prints_the_resumed_iterations(capfd):
    sv = S.gather_2d(seed=3201, n_shots=64, nt=300)
    prob = A.Problem.from_survey(sv)
    _, model = prob.solve_range(sv.data, 1.0, 12, 0, 6)
    capfd.readouterr()
    prob.solve_range(sv.data, 1.0, 12, 6, 12, model_in=model, print_freq=2)
    out = capfd.readouterr().out
    assert "Iteration 0 Residual" not in out
    assert "Iteration 6 Residual" in out and "Iteration 10 Residual" in out
    prob.close()


def test_resume_argument_errors(capfd):
    sv = S.gather_2d(seed=3202, n_shots=48, nt=300)
    prob = A.Problem.from_survey(sv)
    with pytest.raises(RuntimeError):
        prob.solve_range(sv.data, 1.0, 10, 4, 10)  # no model to resume from
    with pytest.raises(RuntimeError):
        prob.solve_range(sv.data, 1.0, 10, 6, 4, model_in=np.zeros(2 * prob.model_size))
    with pytest.raises(RuntimeError):
        prob.solve_range(sv.data, 1.0, 10, 0, 11)
    assert "agd_gpu_solve_range" in capfd.readouterr().err
    prob.close()


def _free_bytes(torch, lib):
    lib.agd_gpu_release_cache()
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _walk_failures(run):
    """Fails allocation 1, 2, ... until a call succeeds; returns the number
    of failing calls."""
    n = 0
    try:
        while True:
            n += 1
            os.environ["AGD_GPU_FAIL_ALLOC"] = str(n)
            try:
                run()
            except RuntimeError:
                continue
            break
    finally:
        os.environ.pop("AGD_GPU_FAIL_ALLOC", None)
    return n - 1


def test_every_allocation_failure_returns_1_and_releases_memory(capfd):
    torch = pytest.importorskip("torch")
    lib = A.load_library(np.float32)
    lib.agd_gpu_release_cache.restype = None
    sv = random_problem(8, wavelets=True)
    kw = dict(wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)

    def deblend():
        return A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                         sv.trace_types, 1.0, 5, 0, sv.data, **kw)

    flat = [d.reshape(-1, d.shape[-1]) for d in sv.data]
    tt_out = [np.where(np.asarray(t) == S.BAD, S.LIVE, t).astype(np.int32)
              for t in sv.trace_types]  # agd_blend takes no bad output traces

    def blend():
        return A.blend(sv.shottimes, sv.channels, sv.trace_types, flat, A.AGDBlendSum,
                       trace_types_out=tt_out)

    ref = deblend()  # loads every module and fills the caches once
    blend()
    free0 = _free_bytes(torch, lib)
    failing = _walk_failures(deblend)
    assert failing >= 10  # the walk went through the problem's allocations
    failing_blend = _walk_failures(blend)
    assert failing_blend >= 5
    free1 = _free_bytes(torch, lib)
    assert abs(free1 - free0) <= 4 << 20
    assert "injected device allocation failure" in capfd.readouterr().err
    # the library still works, with the same result
    for a, b in zip(deblend(), ref):
        assert rel_l2(a, b) <= 1e-6


@pytest.mark.parametrize("print_freq", [0, 2])
def test_non_finite_input_returns_error(print_freq, capfd):
    """A NaN in the host input makes the FP64 residual norm non-finite: the
    call returns 1 (RuntimeError here) with an error message instead of
    writing NaN output, and the library stays usable.  The NaN reaches the
    device only as data; no kernel faults."""
    sv = S.gather_2d(seed=3300, n_shots=48, nt=256, window=(16, 128), n_its=6)
    bad = [d.copy() for d in sv.data]
    bad[0][7, 100] = np.nan
    with pytest.raises(RuntimeError):
        A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                  sv.trace_types, 1.0, 6, print_freq, bad)
    assert "not finite" in capfd.readouterr().err
    inf = [d.copy() for d in sv.data]
    inf[0][3, 50] = np.inf
    prob = A.Problem.from_survey(sv)
    with pytest.raises(RuntimeError):
        prob.solve(inf, 1.0, 6)
    out = prob.solve(sv.data, 1.0, 6)
    prob.close()
    assert all(np.isfinite(o).all() for o in out)
