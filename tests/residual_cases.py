"""Surveys whose printed residual lines are compared with the reference's
(tests/golden/make_residual_fixture.py writes the reference side)."""
from agdeblend_b200 import synthetic as S

CASES = ("gather_2d", "two_volume_3d", "vibroseis_4d")


def make_case(name):
    """(survey, print_freq) of a residual-line case."""
    if name == "gather_2d":
        return S.gather_2d(seed=21, n_shots=96, nt=384, window=(32, 256), n_its=40), 5
    if name == "two_volume_3d":
        return S.two_volume_3d(seed=22, n_ch=8, n_shots=24, nt=300, window=(4, 8, 128),
                               n_its=30), 3
    if name == "vibroseis_4d":
        return S.vibroseis_4d(seed=23, n_sy=4, n_sx=8, n_ch=8, nt=300, window=(4, 4, 4, 64),
                              wavelet_len=40, n_its=20), 4
    raise KeyError(name)
