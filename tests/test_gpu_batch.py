"""Independent problems solved together (agd_deblend_batch,
agd_gpu_batch_create) and problems whose windows fall into several shape
classes (some on the shape-specialised kernels, some on the generic ones).

A batch must leave every problem's data as agd_deblend leaves it for that
problem alone: each problem keeps its step size, initial threshold and
threshold schedule; only the kernel launches are shared."""
import os

import numpy as np
import pytest

import agd_oracle as O
import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from conftest import rel_l2
from golden_io import GOLDEN, sketch
from problems import random_problem

pytestmark = pytest.mark.gpu


def _kw(sv):
    kw = dict(volumes=sv.volumes, window_shapes=sv.window_shapes, coords=sv.coords,
              shottimes=sv.shottimes, channels=sv.channels, trace_types=sv.trace_types,
              data=sv.data)
    if sv.wavelets is not None:
        kw.update(wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)
    return kw


def _single(sv, n_its):
    return A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                     sv.trace_types, 1.0, n_its, 0, sv.data,
                     **({} if sv.wavelets is None else
                        dict(wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)))


def _plan(sv):
    return O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)


def _gathers():
    """Uneven 2-D gathers: window shapes (16,128), (32,256), (64,256) and
    shot counts that do or do not tile the windows."""
    return [S.gather_2d(seed=3100, n_shots=100, nt=512, window=(16, 128)),
            S.gather_2d(seed=3101, n_shots=128, nt=700, window=(32, 256)),
            S.gather_2d(seed=3102, n_shots=150, nt=600, window=(64, 256)),
            S.gather_2d(seed=3103, n_shots=64, nt=512, window=(32, 256)),
            S.gather_2d(seed=3104, n_shots=50, nt=900, window=(16, 128))]


def test_batch_matches_separate_solves():
    gathers = _gathers()
    n_its = 30
    outs = A.deblend_batch([_kw(g) for g in gathers], 1.0, n_its)
    for g, out in zip(gathers, outs):
        ref = _single(g, n_its)
        for o, r in zip(out, ref):
            assert rel_l2(o, r) <= 1e-6


def test_batch_handle_steps_and_solve():
    gathers = _gathers()
    prob = A.Problem.from_batch(gathers)
    steps = prob.steps()
    for g, st in zip(gathers, steps):
        single = A.Problem.from_survey(g)
        assert abs(float(st) - single.stepsize) <= 1e-7 * single.stepsize
        single.close()
    assert prob.info[15] >= 2  # several window classes on the fast kernels
    data = [d for g in gathers for d in g.data]
    out = prob.solve(data, 1.0, 20)
    k = 0
    for g in gathers:
        ref = _single(g, 20)
        for r in ref:
            assert rel_l2(out[k], r) <= 1e-6
            k += 1
    prob.close()


def test_batch_of_random_problems_with_wavelets():
    probs = [random_problem(s, wavelets=True) for s in (8, 13, 22)]
    outs = A.deblend_batch([_kw(p) for p in probs], 1.0, 15)
    for p, out in zip(probs, outs):
        ref = _single(p, 15)
        for o, r in zip(out, ref):
            assert rel_l2(o, r) <= 1e-6


def test_batch_rejects_mixed_wavelets(capfd):
    a = random_problem(8, wavelets=True)
    b = random_problem(9, wavelets=False)
    with pytest.raises(RuntimeError):
        A.deblend_batch([_kw(a), _kw(b)], 1.0, 5)
    assert "all have wavelets" in capfd.readouterr().err


def test_mixed_window_classes_vs_oracle_and_generic():
    """n_shots = 50 with windows of 16 splits into windows of 17 and 16
    samples: the 16-sample windows run the shape-specialised kernels, the
    17-sample ones the generic kernels, in the same operator."""
    sv = S.gather_2d(seed=3105, n_shots=50, nt=600, window=(16, 128))
    prob = A.Problem.from_survey(sv)
    assert prob.info[8] == 2 and 0 < prob.info[16] < prob.info[0]
    plan = _plan(sv)
    rng = np.random.default_rng(3)
    rec = rng.standard_normal(prob.record_size)
    O.apply_mute(plan.cfg, rec)
    x = prob.adjoint(rec)
    x_ref = O.model_to_flat(O.adjoint(plan, rec))
    x_ref = np.stack([x_ref.real, x_ref.imag], -1).reshape(-1)
    assert rel_l2(x, x_ref) <= 1e-5
    y = prob.forward(x_ref)
    y_ref = O.forward(plan, O.flat_to_model(plan, x_ref[0::2] + 1j * x_ref[1::2]))
    assert rel_l2(y, y_ref) <= 1e-5
    out = prob.solve(sv.data, 1.0, 20)
    ref = O.deblend(plan, sv.data, 1.0, 20)
    for o, r in zip(out, ref):
        assert rel_l2(o, r) <= 1e-3
    prob.close()
    old = os.environ.get("AGD_GPU_GENERIC")
    os.environ["AGD_GPU_GENERIC"] = "1"
    try:
        gen = A.Problem.from_survey(sv)
    finally:
        if old is None:
            del os.environ["AGD_GPU_GENERIC"]
        else:
            os.environ["AGD_GPU_GENERIC"] = old
    assert gen.info[8] == 0
    out_g = gen.solve(sv.data, 1.0, 20)
    for a, b in zip(out, out_g):
        assert rel_l2(a, b) <= 1e-5
    gen.close()


def _odd_offset_batch():
    """A gather whose enlarged windows (37, 37 and 36 samples: padded 47,
    47, 45; 5 time windows of 161 bins) have odd model sizes, then a gather
    of 32-sample windows on the shape-specialised kernels, whose models then
    start at odd complex offsets (8-byte but not 16-byte aligned)."""
    a = S.gather_2d(seed=3110, n_shots=78, nt=500, window=(32, 256))
    b = S.gather_2d(seed=3111, n_shots=64, nt=500, window=(32, 256))
    off, odd_fast = 0, 0
    for g in (a, b):
        info, win, bl = A.plan_export(g.volumes, g.n_dims, g.window_shapes, g.coords, g.shapes,
                                      g.shottimes, g.channels, g.trace_types)
        for row in win:
            if row[10] * 5 == row[14] * 4 and off % 2:
                odd_fast += 1
            off += int(row[2]) * int(row[3]) * int(row[14])
    assert odd_fast > 0
    return [a, b]


def test_every_space_candidate_at_odd_model_offsets():
    gathers = _odd_offset_batch()
    refs = [_single(g, 10) for g in gathers]
    probe = A.Problem.from_batch(gathers)
    n = int(max(probe.info[12], probe.info[13]))
    probe.close()
    old = os.environ.get("AGD_GPU_SPACE_VARIANT")
    try:
        for v in range(n):
            os.environ["AGD_GPU_SPACE_VARIANT"] = f"{v},{v}"
            outs = A.deblend_batch([_kw(g) for g in gathers], 1.0, 10)
            for out, ref in zip(outs, refs):
                for o, r in zip(out, ref):
                    assert rel_l2(o, r) <= 1e-5
    finally:
        if old is None:
            os.environ.pop("AGD_GPU_SPACE_VARIANT", None)
        else:
            os.environ["AGD_GPU_SPACE_VARIANT"] = old


def test_uneven_gathers_batch_matches_reference_per_gather():
    """The benchmark's 96 uneven gathers (shots U{100..400}, time
    U{512..2048}, three window shapes), solved together by
    agd_deblend_batch, against the reference float build run separately on
    each gather (tests/golden/make_batch_fixture.py): per gather, SNR
    within 0.05 dB and a 32-projection sketch of the output within 1e-3
    relative difference (an estimate of the relative L2 difference)."""
    ref = np.load(os.path.join(GOLDEN, "uneven_gathers_reference.npz"))
    gathers = S.uneven_gathers(len(ref["snr_db"]), base_seed=int(ref["base_seed"]))
    n_its = int(ref["n_its"])
    for g, c in zip(gathers, ref["input_checksum"]):
        assert g.n_its == n_its
        assert sum(float(np.sum(d.astype(np.float64))) for d in g.data) == \
            pytest.approx(float(c), rel=1e-12)
    outs = A.deblend_batch([_kw(g) for g in gathers], 1.0, n_its)
    k = ref["sketch"].shape[1]
    for i, (g, out) in enumerate(zip(gathers, outs)):
        assert all(np.isfinite(o).all() for o in out), i
        snr = S.snr_db(out, g.truth, g.trace_types)
        assert abs(snr - float(ref["snr_db"][i])) <= 0.05, (i, snr, float(ref["snr_db"][i]))
        sk = sketch(out, k=k)
        rs = ref["sketch"][i]
        assert np.linalg.norm(sk - rs) <= 1e-3 * np.linalg.norm(rs), i
        norm = np.sqrt(sum(float(np.sum(np.asarray(o, np.float64) ** 2)) for o in out))
        assert norm == pytest.approx(float(ref["norm"][i]), rel=1e-3), i
