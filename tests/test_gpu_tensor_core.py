"""The tcgen05 BF16 GEMM (agd_nn_gemm_bf16) against an FP32 product of the
same BF16 operands (torch on the GPU): relative L2 error within 1e-5 (the
tensor cores accumulate in FP32, in another order), on shapes with partial
tiles in M, N and K, with alpha and beta, through the C-ABI.  Products
without split K run on the persistent kernel (tc_gemm_pipe)."""
import ctypes

import numpy as np
import pytest

import agdeblend_b200 as A
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _gemm():
    lib = A.load_library(np.float32)
    fn = lib.agd_nn_gemm_bf16
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 6 + \
        [ctypes.c_float, ctypes.c_float, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


# the last four have more output tiles than the GPU holds CTAs at once, so
# the persistent CTAs walk several tiles (both TMEM accumulators, every
# stage of the ring, one- and many-step K)
@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (200, 100, 72), (1000, 256, 520),
                                   (37, 16, 8), (513, 129, 1024), (76800, 32, 288),
                                   (40000, 64, 576), (70001, 200, 136), (50000, 48, 8)])
def test_tc_gemm_matches_fp32_product(M, N, K):
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    a = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    c0 = torch.randn(M, N, device="cuda", generator=g)
    want = 0.5 * (a.float() @ b.float().T) + 2.0 * c0
    c = c0.clone()
    torch.cuda.synchronize()
    rc = _gemm()(a.data_ptr(), b.data_ptr(), c.data_ptr(), M, N, K, K, K, N, 0.5, 2.0, None)
    assert rc == 0
    assert rel_l2(c.cpu().numpy(), want.cpu().numpy()) <= 1e-5


def test_tc_gemm_rejects_misaligned_k():
    torch = pytest.importorskip("torch")
    a = torch.zeros(16, 12, device="cuda", dtype=torch.bfloat16)
    c = torch.zeros(16, 16, device="cuda")
    assert _gemm()(a.data_ptr(), a.data_ptr(), c.data_ptr(), 16, 16, 12, 12, 12, 16, 1.0, 0.0,
                   None) == 1


def _conv():
    lib = A.load_library(np.float32)
    fn = lib.agd_nn_conv3x3_bf16
    fn.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int,
                                                            ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


# (n, h, w, cin, cout): the halo-tile kernel (w a multiple of 128, cin a
# multiple of 32) with two CTAs per SM - one image row, one-row images, 2
# channel blocks, 8 and 64 output channels, weights at the 36 KB limit, more
# tiles than resident CTAs - and with one CTA per SM - 64 and 128 channels in
# one group, 128 and 96 (a partial second group) in two; the implicit GEMM
# for the rest (w = 64, 256 output channels, 2304-long weight rows, cin = 8)
@pytest.mark.parametrize("n,h,w,cin,cout", [(2, 5, 256, 32, 32), (3, 1, 128, 64, 8),
                                            (1, 4, 384, 32, 64), (2, 3, 128, 64, 32),
                                            (4, 32, 1024, 32, 32), (1, 3, 256, 64, 64),
                                            (1, 3, 128, 64, 128), (2, 2, 128, 128, 128),
                                            (1, 2, 128, 128, 96), (8, 16, 512, 64, 64),
                                            (2, 6, 64, 32, 32), (1, 2, 128, 128, 256),
                                            (1, 2, 128, 256, 128), (2, 4, 256, 8, 16)])
def test_conv3x3_matches_float64(n, h, w, cin, cout):
    """agd_nn_conv3x3_bf16 against a float64 convolution of the same BF16
    values: relative L2 within 1e-5 (FP32 accumulation)."""
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(n * 1000 + h * 100 + w + cin + cout)
    x = torch.randn(n, h, w, cin, generator=g).to(torch.bfloat16)
    wt = torch.randn(cout, 3, 3, cin, generator=g).to(torch.bfloat16)
    want = torch.nn.functional.conv2d(x.double().permute(0, 3, 1, 2),
                                      wt.double().permute(0, 3, 1, 2), padding=1)
    want = want.permute(0, 2, 3, 1).numpy()
    xd, wd = x.cuda(), wt.cuda()
    y = torch.full((n, h, w, cout), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert _conv()(xd.data_ptr(), n, h, w, cin, wd.data_ptr(), cout, y.data_ptr(), None) == 0
    assert rel_l2(y.cpu().numpy().astype(np.float64), want) <= 1e-5
