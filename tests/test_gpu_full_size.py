"""The full benchmark survey (2 volumes of 64 x 128 x 1024, windows
(16, 32, 256), 200 iterations) through agd_deblend on the GPU, against the
reference float (OpenMP) build's output on the same survey recorded in
tests/golden/two_volume_3d_reference.npz (tests/golden/make_full_fixture.py):
its SNR within 0.05 dB and a 64-projection sketch of its 16.8 M output
samples within 1e-3 relative difference."""
import os

import numpy as np
import pytest

import agdeblend_b200 as A
from agdeblend_b200 import synthetic as S
from golden_io import GOLDEN, sketch

pytestmark = pytest.mark.gpu


def test_full_benchmark_survey_matches_reference_output():
    ref = np.load(os.path.join(GOLDEN, "two_volume_3d_reference.npz"))
    sv = S.two_volume_3d()
    checksum = sum(float(np.sum(d.astype(np.float64))) for d in sv.data)
    assert checksum == pytest.approx(float(ref["input_checksum"]), rel=1e-12)
    assert sv.n_its == int(ref["n_its"])
    out = A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes, sv.channels,
                    sv.trace_types, sv.initial_factor, sv.n_its, 0, sv.data)
    assert all(np.isfinite(o).all() for o in out)
    snr = S.snr_db(out, sv.truth, sv.trace_types)
    assert abs(snr - float(ref["snr_db"])) <= 0.05
    sk = sketch(out)
    assert np.linalg.norm(sk - ref["sketch"]) <= 1e-3 * np.linalg.norm(ref["sketch"])
    norm = np.sqrt(sum(float(np.sum(np.asarray(o, np.float64) ** 2)) for o in out))
    assert norm == pytest.approx(float(ref["norm"]), rel=1e-3)
