"""The algebra of the line-DFT space kernels (agdeblend_b200/csrc/line_dft.cuh),
restated in numpy and checked against the DFT definition (np.fft) on the
CPU: the forward pairs inputs j and P - j, the adjoint pairs outputs k and
P - k, both from tables of cos / sin(2 pi (j k mod P) / P) built as the
engine builds them.  The GPU parity of the kernels themselves is in
test_gpu_line_dft.py."""
import numpy as np
import pytest


def _tables(P, rows, j0, kout):
    j = np.arange(rows)[:, None] + j0
    k = np.arange(kout)[None, :]
    ang = 2.0 * np.pi * ((j * k) % P) / P
    return np.cos(ang), np.sin(ang)


def _forward(x, P, L):
    """Inverse DFT of each line (unnormalised), first L outputs."""
    H = (P - 1) // 2
    c, s = _tables(P, H, 1, L)
    j = np.arange(1, H + 1)
    ssum = x[:, j] + x[:, P - j]
    sdif = x[:, j] - x[:, P - j]
    y = x[:, :1] + (ssum @ c) + 1j * (sdif @ s)
    if P % 2 == 0:
        y = y + x[:, P // 2:P // 2 + 1] * ((-1.0) ** np.arange(L))
    return y


def _adjoint(x, P, L):
    """Forward DFT of each line zero-padded from L to P, all P outputs."""
    kout = P // 2 + 1
    c, s = _tables(P, L, 0, kout)
    A = x @ c
    B = x @ s
    y = np.zeros((x.shape[0], P), complex)
    y[:, :kout] = A - 1j * B
    k = np.arange(1, kout)
    k = k[P - k != k]
    y[:, P - k] = A[:, k] + 1j * B[:, k]
    return y


@pytest.mark.parametrize("P,L", [(20, 16), (22, 17), (42, 33), (43, 34), (83, 66), (84, 67),
                                 (89, 71), (127, 101), (128, 102)])
def test_paired_forms_match_the_dft(P, L):
    rng = np.random.default_rng(P * 1000 + L)
    x = rng.standard_normal((5, P)) + 1j * rng.standard_normal((5, P))
    y = _forward(x, P, L)
    ref = np.fft.ifft(x, axis=1)[:, :L] * P
    assert np.max(np.abs(y - ref)) <= 1e-11 * np.max(np.abs(ref))
    z = rng.standard_normal((5, L)) + 1j * rng.standard_normal((5, L))
    g = _adjoint(z, P, L)
    ref = np.fft.fft(np.pad(z, ((0, 0), (0, P - L))), axis=1)
    assert np.max(np.abs(g - ref)) <= 1e-11 * np.max(np.abs(ref))


def test_forward_and_adjoint_are_adjoint():
    # <F x, z> = <x, F^H z> with F the cropped inverse DFT and F^H the padded
    # forward DFT (the pair the kernels apply in the operator and its adjoint)
    rng = np.random.default_rng(7)
    P, L = 83, 66
    x = rng.standard_normal((3, P)) + 1j * rng.standard_normal((3, P))
    z = rng.standard_normal((3, L)) + 1j * rng.standard_normal((3, L))
    lhs = np.vdot(z, _forward(x, P, L))
    rhs = np.vdot(_adjoint(z, P, L), x)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
