"""CPU model of the split-BF16 tensor-core space kernels (space_tc.cuh), run
before any GPU: the same row / k index maps of the three passes, the same
real matrices on interleaved (re, im) values and the same shared-memory
operand offsets.

  * the composed passes equal the space part of the FK operator: the
    forward crop(inverse DFT) of a padded 20^3 plane and the adjoint
    forward DFT of the zero-padded 16^3 plane (numpy FFT, float64);
  * every (row, k) an epilogue or the conversion writes maps to a distinct
    operand byte offset inside the operand buffer, and every byte an MMA
    descriptor can read (128 rows x 2 chunks per K step, 16 row groups per
    tile) lies inside the buffer of the tiles the pass issues;
  * the BF16 split keeps about 16 significant bits (hi + lo vs the value).
"""
import numpy as np
import pytest

P, L = 20, 16
LBO = 144


def sbo(kch):
    return (kch - 1) * LBO + 128


def offset(row, k, kch):
    return (row // 8) * sbo(kch) + (k // 8) * LBO + (row % 8) * 16 + (k % 8) * 2


def real_matrix(w):
    """Real matrix acting on interleaved (re, im) of a complex matrix w
    (outputs x inputs): B[2i+a][2j+b]."""
    n, m = w.shape
    b = np.zeros((2 * n, 2 * m))
    b[0::2, 0::2] = w.real
    b[0::2, 1::2] = -w.imag
    b[1::2, 0::2] = w.imag
    b[1::2, 1::2] = w.real
    return b


def interleave(x):
    out = np.empty(x.shape[:-1] + (2 * x.shape[-1],))
    out[..., 0::2] = x.real
    out[..., 1::2] = x.imag
    return out


def deinterleave(v):
    return v[..., 0::2] + 1j * v[..., 1::2]


def fwd_model(x):
    """space_fwd_tc: X[a][b][c] (P^3) -> Z[n0][n1][n2] (L^3)."""
    n = np.arange(L)[:, None]
    k = np.arange(P)[None, :]
    B = real_matrix(np.exp(2j * np.pi * n * k / P))  # 2L x 2P
    # pass 1 operand: rows (a, b) = a P + b, k = 2 c
    A = np.zeros((P * P, 2 * P))
    for e in range(P ** 3):
        r, c = divmod(e, P)
        A[r, 2 * c: 2 * c + 2] = [x.flat[e].real, x.flat[e].imag]
    D = A @ B.T  # rows (a, b), columns 2 n2 + (re, im)
    A2 = np.zeros((L * P, 2 * P))
    for r in range(P * P):
        ra, rb = divmod(r, P)
        for n2 in range(L):
            A2[n2 * P + ra, 2 * rb: 2 * rb + 2] = D[r, 2 * n2: 2 * n2 + 2]
    D2 = A2 @ B.T  # rows (n2, a), columns n1
    A3 = np.zeros((L * L, 2 * P))
    for r in range(L * P):
        rn2, ra = divmod(r, P)
        for n1 in range(L):
            A3[n1 * L + rn2, 2 * ra: 2 * ra + 2] = D2[r, 2 * n1: 2 * n1 + 2]
    D3 = A3 @ B.T  # rows (n1, n2), columns n0
    z = np.zeros(L ** 3, complex)
    for r in range(L * L):
        for n0 in range(L):
            z[n0 * L * L + r] = D3[r, 2 * n0] + 1j * D3[r, 2 * n0 + 1]
    return z.reshape(L, L, L)


def adj_model(g):
    """space_adj_tc: G[n0][n1][n2] (L^3) -> X[a][b][c] (P^3)."""
    k = np.arange(P)[:, None]
    n = np.arange(L)[None, :]
    B = real_matrix(np.exp(-2j * np.pi * n * k / P))  # 2P x 2L
    A = np.zeros((L * L, 2 * L))
    for e in range(L ** 3):
        r, c = divmod(e, L)
        A[r, 2 * c: 2 * c + 2] = [g.flat[e].real, g.flat[e].imag]
    D = A @ B.T  # rows (n0, n1), columns c
    A2 = np.zeros((P * L, 2 * L))
    for r in range(L * L):
        rn0, rn1 = divmod(r, L)
        for c in range(P):
            A2[c * L + rn0, 2 * rn1: 2 * rn1 + 2] = D[r, 2 * c: 2 * c + 2]
    D2 = A2 @ B.T  # rows (c, n0), columns b
    A3 = np.zeros((P * P, 2 * L))
    for r in range(P * L):
        rc, rn0 = divmod(r, L)
        for b in range(P):
            A3[b * P + rc, 2 * rn0: 2 * rn0 + 2] = D2[r, 2 * b: 2 * b + 2]
    D3 = A3 @ B.T  # rows (b, c), columns a
    x = np.zeros(P ** 3, complex)
    for r in range(P * P):
        for a in range(P):
            x[a * P * P + r] = D3[r, 2 * a] + 1j * D3[r, 2 * a + 1]
    return x.reshape(P, P, P)


def test_forward_passes_equal_cropped_inverse_dft():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((P, P, P)) + 1j * rng.standard_normal((P, P, P))
    want = (np.fft.ifftn(x) * P ** 3)[:L, :L, :L]
    got = fwd_model(x)
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()


def test_adjoint_passes_equal_padded_forward_dft():
    rng = np.random.default_rng(1)
    g = rng.standard_normal((L, L, L)) + 1j * rng.standard_normal((L, L, L))
    pad = np.zeros((P, P, P), complex)
    pad[:L, :L, :L] = g
    want = np.fft.fftn(pad)
    got = adj_model(g)
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    # the adjoint is the conjugate transpose of the forward
    rng2 = np.random.default_rng(2)
    x = rng2.standard_normal((P, P, P)) + 1j * rng2.standard_normal((P, P, P))
    assert np.vdot(fwd_model(x), g) == pytest.approx(np.vdot(x, got), rel=1e-12)


@pytest.mark.parametrize("kch,k_used,rows_by_pass,smem_end", [
    # forward: K 48 (40 used); A hi at 0, A lo at 50 row groups; the barrier
    # sits where the last tile of A lo ends (no MMA reads past it)
    (6, 2 * P, [P * P, L * P, L * L], 2 * 50 * sbo(6) + 14 * sbo(6)),
    # adjoint: K 32; the model plane (64000 bytes) is staged over the A area,
    # the B matrices start at 64000
    (4, 2 * L, [L * L, P * L, P * P], 64000),
])
def test_operand_offsets_distinct_and_in_bounds(kch, k_used, rows_by_pass, smem_end):
    a_bytes = (P * P // 8) * sbo(kch)  # one operand (hi or lo): the P * P rows
    for rows in rows_by_pass:
        offs = np.array([offset(r, k, kch) for r in range(rows) for k in range(0, k_used, 2)])
        assert offs.min() >= 0 and offs.max() + 4 <= a_bytes
        assert len(np.unique(offs)) == offs.size
        # bytes an MMA can read: tiles of the pass, K steps of 2 chunks, from
        # A lo (the later of the two operands)
        tiles = (rows + 127) // 128
        for t in range(tiles):
            for s in range(kch // 2):
                start = a_bytes + t * 16 * sbo(kch) + s * 2 * LBO
                last = start + 15 * sbo(kch) + LBO + 128
                assert last <= smem_end
    # the padding chunk (forward: k 40..47) is never written by an epilogue
    if kch * 8 > k_used:
        pad = {offset(r, k, kch) for r in range(P * P) for k in range(k_used, kch * 8, 2)}
        used = {offset(r, k, kch) for r in range(P * P) for k in range(0, k_used, 2)}
        assert not pad & used


def _bf16(v):
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def test_bf16_split_keeps_sixteen_bits():
    rng = np.random.default_rng(3)
    v = rng.standard_normal(100000).astype(np.float32).astype(np.float64)
    hi = _bf16(v)
    lo = _bf16(v - hi)
    assert np.max(np.abs(v - hi - lo) / np.abs(v)) <= 2.0 ** -16
