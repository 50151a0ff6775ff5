"""Index maps of the prime-factor (Good-Thomas) transforms, restated in numpy
and checked against the DFT definition on the CPU.

* The wavelet stage (agdeblend_b200/csrc/wavelet_fast.cuh): sample t goes
  to the dense position with coordinates t mod f_i; plain DFTs along every
  axis then leave frequency k at coordinates k (C / f_i)^-1 mod f_i, and the
  inverse passes return the sample layout.
* The register DFTs (agdeblend_b200/csrc/fast.cuh dft_pfa): for coprime
  N1, N2, inputs n = (n1 N2 + n2 N1) mod N through an N1-point then an
  N2-point DFT give X_k at the k with k = k1 (mod N1), k = k2 (mod N2).
The GPU kernels' parity is tested in the test_gpu_* files."""
import numpy as np
import pytest


def _dense_maps(N, f):
    g = [1] * len(f)
    for i in range(len(f) - 2, -1, -1):
        g[i] = g[i + 1] * f[i + 1]
    inv = [pow(N // fi, -1, fi) if fi > 1 else 0 for fi in f]
    qmap = np.array([sum((t % fi) * gi for fi, gi in zip(f, g)) for t in range(N)])
    kpos = np.array([sum((k * iv % fi) * gi for fi, gi, iv in zip(f, g, inv))
                     for k in range(N)])
    return qmap, kpos


@pytest.mark.parametrize("N,f", [(2431, [11, 13, 17]), (30, [2, 3, 5]), (16, [16]), (17, [17]),
                                 (1260, [4, 9, 5, 7]), (4 * 11 * 13, [4, 11, 13])])
def test_dense_prime_factor_layout(N, f):
    qmap, kpos = _dense_maps(N, f)
    assert sorted(qmap) == list(range(N)) and sorted(kpos) == list(range(N))
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    a = np.zeros(N, complex)
    a[qmap] = x
    a = a.reshape(f)
    for ax in range(len(f)):
        a = np.fft.fft(a, axis=ax)
    X = a.reshape(-1)[kpos]
    ref = np.fft.fft(x)
    assert np.max(np.abs(X - ref)) <= 1e-12 * np.max(np.abs(ref))
    b = a
    for ax in range(len(f)):
        b = np.fft.ifft(b, axis=ax)
    assert np.max(np.abs(b.reshape(-1)[qmap] - x)) <= 1e-12 * np.max(np.abs(x))


def _crt(k1, k2, n1, n2):
    k = k2
    while k % n1 != k1:
        k += n2
    return k


@pytest.mark.parametrize("N1,N2", [(4, 5), (8, 5), (2, 5), (4, 3), (16, 5), (8, 3), (3, 5)])
@pytest.mark.parametrize("inverse", [False, True])
def test_register_prime_factor_split(N1, N2, inverse):
    N = N1 * N2
    rng = np.random.default_rng(N1 * 100 + N2)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    sign = 1.0 if inverse else -1.0
    dft = lambda v: np.exp(sign * 2j * np.pi * np.outer(np.arange(len(v)), np.arange(len(v)))
                           / len(v)) @ v
    a = np.zeros((N1, N2), complex)
    for n2 in range(N2):
        a[:, n2] = dft(np.array([x[(n1 * N2 + n2 * N1) % N] for n1 in range(N1)]))
    v = np.zeros(N, complex)
    for k1 in range(N1):
        t = dft(a[k1, :])
        for k2 in range(N2):
            v[_crt(k1, k2, N1, N2)] = t[k2]
    ref = dft(x)
    assert np.max(np.abs(v - ref)) <= 1e-12 * np.max(np.abs(ref))
