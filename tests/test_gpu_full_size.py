"""Benchmark-shaped surveys through agd_deblend on the GPU, against the
reference float (OpenMP) build's output on the same survey recorded in
tests/golden/<workload>_reference.npz (tests/golden/make_full_fixture.py):
the SNR within 0.05 dB, a 64-projection sketch of the output within 1e-3
relative difference, and the output's L2 norm within 1e-3.

  two_volume_3d       2 x 64 ch x 128 shots x 1024, windows (16, 32, 256),
                      the full 200 iterations (16.8 M output samples);
  vibroseis_4d        32 sY x 64 sX x 32 ch x 2048 with the 256-sample sweep,
                      windows (16, 16, 16, 256), model 10.4 GB: the
                      reference's n_its = 5 run (its 150 iterations take it
                      hours on a CPU);
  vibroseis_4d_small  16 sY x 32 sX x 32 ch x 2048, the full 150 iterations.
"""
import os

import numpy as np
import pytest

import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from golden_io import GOLDEN, sketch

pytestmark = pytest.mark.gpu

SURVEYS = {
    "two_volume_3d": lambda: S.two_volume_3d(),
    "vibroseis_4d": lambda: S.vibroseis_4d(seed=1002),
    "vibroseis_4d_small": lambda: S.vibroseis_4d(seed=1002, n_sy=16, n_sx=32),
}


@pytest.mark.parametrize("name", list(SURVEYS))
def test_full_survey_matches_reference_output(name):
    path = os.path.join(GOLDEN, f"{name}_reference.npz")
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated")
    ref = np.load(path)
    sv = SURVEYS[name]()
    checksum = sum(float(np.sum(d.astype(np.float64))) for d in sv.data)
    assert checksum == pytest.approx(float(ref["input_checksum"]), rel=1e-12)
    n_its = int(ref["n_its"])
    kw = {}
    if sv.wavelets is not None:
        kw = dict(wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)
    out = A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                    sv.trace_types, sv.initial_factor, n_its, 0, sv.data, **kw)
    assert all(np.isfinite(o).all() for o in out)
    snr = S.snr_db(out, sv.truth, sv.trace_types)
    assert abs(snr - float(ref["snr_db"])) <= 0.05, (snr, float(ref["snr_db"]))
    sk = sketch(out)
    assert np.linalg.norm(sk - ref["sketch"]) <= 1e-3 * np.linalg.norm(ref["sketch"])
    norm = np.sqrt(sum(float(np.sum(np.asarray(o, np.float64) ** 2)) for o in out))
    assert norm == pytest.approx(float(ref["norm"]), rel=1e-3)
