"""The float64 network oracle (oracle/nn_oracle.py) against itself: its
hand-written backpropagation equals central finite differences of its loss
(float64, no BF16 rounding), with one and with three input channels, and
its parameter count is the CUDA network's (1,162,945 for base 32 channels
and one input channel)."""
import numpy as np
import pytest

import nn_oracle as N


def test_param_count_base32():
    assert N.param_count(32) == 1162945


def test_param_count_three_input_channels():
    # only the first layer's weights grow: 9 x 3 x 32 instead of 9 x 1 x 32
    assert N.param_count(32, 3) == 1162945 + 9 * 2 * 32


@pytest.mark.parametrize("in_ch", [1, 3])
def test_backprop_matches_finite_differences(in_ch):
    rng = np.random.default_rng(0)
    base = 2
    params = N.init_params(base, seed=1, in_ch=in_ch)
    x = rng.standard_normal((2, 8, 16, in_ch))
    target = x[..., 0] + 0.3 * rng.standard_normal(x.shape[:3])
    net = N.Net(base, params, bf16_like_gpu=False, in_ch=in_ch)
    loss, g = net.loss_grad(x, target)
    idx = rng.choice(params.size, 60, replace=False)
    h = 1e-6
    for i in idx:
        p1 = params.copy()
        p1[i] += h
        p2 = params.copy()
        p2[i] -= h
        l1 = N.Net(base, p1, False, in_ch).loss_grad(x, target)[0]
        l2 = N.Net(base, p2, False, in_ch).loss_grad(x, target)[0]
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (i, fd, g[i])


def test_neighbour_lines_channel_order():
    """warmstart.neighbour_lines: channel 0 the line itself, then the lines at
    offsets -1, +1 (clamped at the edges) along the neighbour axis - the
    order agd_gpu_solve_learned gathers on the device."""
    from agdeblend_b200.warmstart import neighbour_lines

    v = np.arange(3 * 4 * 2 * 5, dtype=np.float32).reshape(3, 4, 2, 5)  # (sY, sX, ch, t)
    x = neighbour_lines(v, 1, 0, 1)  # lines along sX, neighbours along sY
    assert x.shape == (3 * 2, 4, 5, 3)
    lines = np.moveaxis(v, 1, 2).reshape(-1, 4, 5)
    for sy in range(3):
        for ch in range(2):
            i = sy * 2 + ch
            assert np.array_equal(x[i, ..., 0], lines[i])
            assert np.array_equal(x[i, ..., 1], lines[max(sy - 1, 0) * 2 + ch])
            assert np.array_equal(x[i, ..., 2], lines[min(sy + 1, 2) * 2 + ch])
