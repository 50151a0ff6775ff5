"""Shared test set-up: the `gpu` marker, import paths and small surveys."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="session")
def small_surveys():
    from agdeblend_b200 import synthetic as S

    return {
        "gather_2d": S.gather_2d(seed=11, n_shots=64, nt=300, window=(16, 128), n_its=30),
        "two_volume_3d": S.two_volume_3d(seed=12, n_ch=16, n_shots=32, nt=300,
                                         window=(8, 16, 128), n_its=30),
        "vibroseis_4d": S.vibroseis_4d(seed=13, n_sy=4, n_sx=8, n_ch=8, nt=300,
                                       window=(4, 4, 4, 64), wavelet_len=40, n_its=20),
    }
