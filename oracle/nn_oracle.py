"""Test infrastructure only: float64 numpy restatement of the warm-start
network of agdeblend_b200/csrc/nn.cu (the checker of its forward pass and of
its gradients; the reference has no network - its solver starts from a zero
model, src/model.c:1160-1185).

Same graph and parameter layout as the CUDA network: 4 levels (channels c,
2c, 4c, 8c), 3 x 3 convolutions with padding 1 (weights [cout][ky][kx][cin]
then biases [cout] per layer), ReLU, 2 x 2 average pooling, nearest 2x
upsampling with additive skips, output = input + last convolution, loss =
mean squared error.  With bf16=True the values the CUDA network feeds to
its tensor cores are rounded to BF16 at the same points (weights, layer
inputs and outputs, backward dZ); every sum is float64.  backward() is
hand-written backpropagation, checked against finite differences in float64.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def architecture(c, in_ch=1):
    """Layers (cin, cout, relu) in parameter order and the op list:
    ("conv", layer, in, out) | ("pool", in, out) | ("up", low, skip, out);
    in_ch input channels."""
    layers, ops, chans = [], [], [in_ch]

    def tensor(ch):
        chans.append(ch)
        return len(chans) - 1

    def conv(x, cout, relu=True):
        layers.append((chans[x], cout, relu))
        o = tensor(cout)
        ops.append(("conv", len(layers) - 1, x, o))
        return o

    def pool(x):
        o = tensor(chans[x])
        ops.append(("pool", x, o))
        return o

    def up(low, skip):
        o = tensor(chans[skip])
        ops.append(("up", low, skip, o))
        return o

    s1 = conv(conv(0, c), c)
    s2 = conv(conv(pool(s1), 2 * c), 2 * c)
    s3 = conv(conv(pool(s2), 4 * c), 4 * c)
    bn = conv(conv(pool(s3), 8 * c), 4 * c)
    d3 = conv(conv(up(bn, s3), 4 * c), 2 * c)
    d2 = conv(conv(up(d3, s2), 2 * c), c)
    conv(conv(up(d2, s1), c), 1, relu=False)
    return layers, ops


def param_count(c, in_ch=1):
    return sum(9 * ci * co + co for ci, co, _ in architecture(c, in_ch)[0])


def _split(params, layers):
    out, off = [], 0
    for ci, co, _ in layers:
        w = params[off: off + 9 * ci * co].reshape(co, 3, 3, ci)
        off += 9 * ci * co
        b = params[off: off + co]
        off += co
        out.append((w, b))
    return out


def im2col(x):
    """x (n, h, w, c) -> (n h w, 9 c), k = (ky 3 + kx) c + ci."""
    n, h, w, c = x.shape
    p = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    cols = [p[:, ky: ky + h, kx: kx + w, :] for ky in range(3) for kx in range(3)]
    return np.concatenate(cols, axis=-1).reshape(n * h * w, 9 * c)


def col2im(dcol, shape):
    n, h, w, c = shape
    d = dcol.reshape(n, h, w, 9, c)
    dp = np.zeros((n, h + 2, w + 2, c))
    for ky in range(3):
        for kx in range(3):
            dp[:, ky: ky + h, kx: kx + w, :] += d[:, :, :, ky * 3 + kx, :]
    return dp[:, 1: h + 1, 1: w + 1, :]


def _pool(x):
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def _unpool(d):
    return 0.25 * np.repeat(np.repeat(d, 2, axis=1), 2, axis=2)


def _up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def _down_sum(d):
    n, h, w, c = d.shape
    return d.reshape(n, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4))


class Net:
    def __init__(self, base, params, bf16_like_gpu=True, in_ch=1):
        self.in_ch = in_ch
        self.layers, self.ops = architecture(base, in_ch)
        self.params = np.asarray(params, np.float64)
        self.q = bf16 if bf16_like_gpu else (lambda a: np.asarray(a, np.float64))
        self.wb = _split(self.params, self.layers)

    def forward(self, x):
        """x (n, h, w), or (n, h, w, in_ch) -> network output (n, h, w) =
        channel 0 + the last convolution; keeps what backward needs."""
        q = self.q
        x = np.asarray(x, np.float64)
        if x.ndim == 3:
            x = x[..., None]
        assert x.shape[3] == self.in_ch
        t = {0: q(x)}
        self.cols = {}
        last = None
        for op in self.ops:
            if op[0] == "conv":
                li, a, o = op[1:]
                wgt, b = self.wb[li]
                relu = self.layers[li][2]
                col = im2col(t[a])
                self.cols[li] = col
                z = col @ q(wgt.reshape(wgt.shape[0], -1)).T + b
                if relu:
                    z = np.maximum(z, 0.0)
                shp = t[a].shape[:3] + (wgt.shape[0],)
                if li == len(self.layers) - 1:
                    last = z.reshape(shp)
                t[o] = q(z.reshape(shp))
            elif op[0] == "pool":
                t[op[2]] = q(_pool(t[op[1]]))
            else:
                t[op[3]] = q(_up(t[op[1]]) + t[op[2]])
        self.t = t
        self.x = x
        self.out = self.x[..., 0] + last[..., 0]
        return self.out

    def loss_grad(self, x, target):
        """(loss, gradient of the loss with respect to params)."""
        q = self.q
        out = self.forward(x)
        P = out.size
        e = out - target
        loss = float(np.sum(e * e) / P)
        g = {k: np.zeros_like(v) for k, v in self.t.items()}
        last_t = self.ops[-1][3]
        g[last_t][..., 0] = 2.0 * e / P
        grads = [None] * len(self.layers)
        for op in reversed(self.ops):
            if op[0] == "conv":
                li, a, o = op[1:]
                wgt, b = self.wb[li]
                relu = self.layers[li][2]
                y = self.t[o]
                dy = g[o]
                dz = np.where(y > 0, dy, 0.0) if relu else dy
                dz = q(dz).reshape(-1, wgt.shape[0])
                dw = dz.T @ self.cols[li]
                db = dz.sum(axis=0)
                grads[li] = (dw.reshape(wgt.shape), db)
                if a != 0:
                    dcol = dz @ q(wgt.reshape(wgt.shape[0], -1))
                    g[a] += col2im(dcol, self.t[a].shape)
            elif op[0] == "pool":
                g[op[1]] += _unpool(g[op[2]])
            else:
                g[op[1]] += _down_sum(g[op[3]])
                g[op[2]] += g[op[3]]
        flat = []
        for dw, db in grads:
            flat.append(dw.reshape(-1))
            flat.append(db)
        return loss, np.concatenate(flat)


def init_params(base, seed=0, in_ch=1):
    """A float64 parameter vector of the layout above (He-normal weights,
    small random biases)."""
    rng = np.random.default_rng(seed)
    layers, _ = architecture(base, in_ch)
    out = []
    for ci, co, _ in layers:
        out.append(rng.standard_normal(9 * ci * co) * np.sqrt(2.0 / (9 * ci)))
        out.append(0.01 * rng.standard_normal(co))
    return np.concatenate(out)
