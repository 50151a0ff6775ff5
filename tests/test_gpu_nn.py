"""The warm-start network's tensor-core forward and backward passes against
the float64 oracle (oracle/nn_oracle.py, which rounds to BF16 where the GPU
feeds its tensor cores, and whose backpropagation is itself checked against
finite differences): output, loss and every parameter gradient on small
shapes; then a short training run lowers the loss.

Tolerances: for base 4 and 8 channels (sums of at most 576 products) output,
loss and gradient within 1e-5 relative: only the FP32 summation order
differs.  For the full network (base 32, sums of up to 2304 products) a sum
that lands on the other side of a BF16 rounding boundary moves a value by
2^-8, and such moves compound over the 14 layers: output and loss within
2e-2, gradient within 5e-2 relative L2 with cosine similarity above 0.999.
The base-8 network with three input channels takes the second tolerance
too: one of its first-layer sums (27 products, FP32 on the CUDA cores)
crosses such a boundary on this input (output 7.9e-4, gradient 1.5e-3 from
the oracle, cosine 0.999999)."""
import numpy as np
import pytest

import nn_oracle as N
from agdeblend_b200.nn import WarmStartNet
from conftest import rel_l2

pytestmark = pytest.mark.gpu


# (base, n, h, w, input channels): one channel, and three (a line and its
# two neighbours, as the vibroseis warm start feeds them)
@pytest.mark.parametrize("base,n,h,w,in_ch", [(4, 2, 16, 32, 1), (8, 3, 8, 64, 1),
                                              (32, 2, 32, 256, 1), (4, 2, 16, 32, 3),
                                              (8, 2, 8, 64, 3)])
def test_forward_and_gradients_match_oracle(base, n, h, w, in_ch):
    net = WarmStartNet(base, seed=base, in_channels=in_ch)
    assert net.n_params == N.param_count(base, in_ch)
    rng = np.random.default_rng(base + n)
    # non-trivial weights everywhere (the network's own last layer starts small)
    p = N.init_params(base, seed=3, in_ch=in_ch).astype(np.float32)
    net.set_params(p)
    shape = (n, h, w) if in_ch == 1 else (n, h, w, in_ch)
    x = rng.standard_normal(shape).astype(np.float32)
    x0 = x if in_ch == 1 else x[..., 0]
    t = (x0 + 0.5 * rng.standard_normal(x0.shape)).astype(np.float32)
    ora = N.Net(base, p.astype(np.float64), bf16_like_gpu=True, in_ch=in_ch)
    loss_o, g_o = ora.loss_grad(x.astype(np.float64), t.astype(np.float64))
    exact = base <= 8 and (in_ch == 1 or base == 4)
    tol_out, tol_grad = (1e-5, 1e-5) if exact else (2e-2, 5e-2)
    y = net.forward(x)
    err_out = rel_l2(y, ora.out)
    loss, g = net.loss_grad(x, t)
    err = rel_l2(g, g_o)
    cos = float(np.dot(g.astype(np.float64), g_o) / np.linalg.norm(g) / np.linalg.norm(g_o))
    print(f"base {base}: output rel L2 {err_out:.2e}, loss {loss:.6e} vs {loss_o:.6e}, "
          f"gradient rel L2 {err:.2e}, cosine {cos:.6f}")
    assert err_out <= tol_out
    assert abs(loss - loss_o) <= tol_out * loss_o
    assert err <= tol_grad and cos >= 0.999
    net.close()


def test_training_lowers_the_loss():
    rng = np.random.default_rng(9)
    n, h, w = 64, 16, 64
    # a task the network can learn quickly: remove a fixed spike pattern
    clean = np.cumsum(rng.standard_normal((n, h, w)), axis=2).astype(np.float32)
    clean /= np.std(clean)
    noisy = clean.copy()
    noisy[:, ::4, ::8] += 2.0
    net = WarmStartNet(8, seed=1)
    losses = net.train(noisy, clean, batch=16, epochs=30, lr=2e-3)
    assert losses[-1] < 0.3 * losses[0]
    net.close()


def test_training_is_deterministic():
    """Two trainings from the same seed on the same data end with identical
    parameters: the split-K weight gradients sum their partial products in
    a fixed order (no atomics)."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal((64, 16, 64, 3)).astype(np.float32)
    t = (x[..., 0] + 0.3 * rng.standard_normal((64, 16, 64))).astype(np.float32)
    params = []
    for _ in range(2):
        net = WarmStartNet(8, seed=2, in_channels=3)
        net.train(x, t, batch=16, epochs=2, lr=1e-3, seed=4)
        params.append(net.params())
        net.close()
    assert np.array_equal(params[0], params[1])
