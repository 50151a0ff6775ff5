"""Learned warm start of the deblending solver.

The network (agdeblend_b200.nn.WarmStartNet, a convolutional encoder-decoder
run on the tensor cores) maps 2-D gathers of pseudo-deblended data (traces x
time samples, each normalised by its RMS) to an estimate of the deblended
data.  The solver then starts from the model that reproduces that estimate
(agd_gpu_solve_warm) and runs only the tail of the plain method's threshold
schedule.  The plain method is unchanged and decides the result: the warm
start only changes where its iterations begin.

Training pairs are made by the plain method itself: seeded synthetic 2-D
receiver gathers (agdeblend_b200.synthetic.gather_2d, 128 shots x 512
samples, base seed 4000) deblended by the GPU solver, cut into 32 x 256
windows of (pseudo-deblended input, deblended output).
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_int

import numpy as np

from . import capi, load_library
from . import synthetic as S
from .nn import WarmStartNet

TRAIN_SEED = 4000


def source_axes(shape, shottimes) -> list:
    """Space axes of a patch along which shot times change, in order of
    their mean shot-time step between neighbouring traces, smallest first
    (the last space axis if none changes): the axes, and their order, of
    the receiver-gather lines agd_gpu_solve_learned cuts on the device."""
    st = np.asarray(shottimes, np.float64).reshape(shape[:-1])
    found = []
    for ax in range(len(shape) - 1):
        if shape[ax] < 2:
            continue
        d = float(np.mean(np.abs(np.diff(st, axis=ax))))
        if d > 0:
            found.append((d, ax))
    found.sort()
    return [ax for _, ax in found] or [len(shape) - 2]


def to_images(patch, axis):
    """(images [n][traces][time], restore) of one patch: every line along
    `axis` becomes one image."""
    a = np.moveaxis(np.asarray(patch, np.float32), axis, -2)
    lead = a.shape[:-2]
    imgs = a.reshape(-1, a.shape[-2], a.shape[-1])

    def restore(out):
        return np.moveaxis(out.reshape(lead + out.shape[-2:]), -2, axis)

    return imgs, restore


def _pad8(n):
    return (n + 7) // 8 * 8


def infer(net: WarmStartNet, images, max_pixels: int = 1 << 23):
    """Network estimate of each image ([n][h][w], or [n][h][w][c] with the
    image in channel 0 and its neighbours after it), normalised in and out
    by the RMS of channel 0; sides zero-padded to multiples of 8."""
    imgs = np.asarray(images, np.float32)
    if imgs.ndim == 3:
        imgs = imgs[..., None]
    n, h, w, c = imgs.shape
    rms = np.sqrt(np.mean(imgs[..., 0].astype(np.float64) ** 2, axis=(1, 2)))
    rms[rms == 0] = 1.0
    hp, wp = _pad8(h), _pad8(w)
    x = np.zeros((n, hp, wp, c), np.float32)
    x[:, :h, :w] = imgs / rms[:, None, None, None]
    if c == 1:
        x = x[..., 0]
    out = np.empty((n, hp, wp), np.float32)
    step = max(1, max_pixels // (hp * wp))
    for i in range(0, n, step):
        out[i: i + step] = net.forward(x[i: i + step])
    return out[:, :h, :w] * rms[:, None, None].astype(np.float32)


def estimate(net: WarmStartNet, sv):
    """Network estimate of the deblended data of every patch of a survey,
    made on the host as agd_gpu_solve_learned makes it on the device: with
    one input channel the mean of the estimates from the lines along every
    source axis; with 2 k + 1 channels the estimate from the lines along
    the slowest source axis, each with its neighbours along the next faster
    one (neighbour_lines; the line itself where there is no other)."""
    est = []
    for d, st in zip(sv.data, sv.shottimes):
        axes = source_axes(d.shape, st)
        if net.in_channels == 1:
            outs = []
            for ax in axes:
                imgs, restore = to_images(d, ax)
                outs.append(restore(infer(net, imgs)))
            est.append(np.mean(outs, axis=0).astype(np.float32))
            continue
        k = (net.in_channels - 1) // 2
        line = axes[-1]
        imgs, restore = to_images(d, line)
        if len(axes) > 1:
            x = neighbour_lines(d, line, axes[-2], k)
        else:
            x = np.repeat(imgs[..., None], net.in_channels, axis=-1)
        est.append(restore(infer(net, x)).astype(np.float32))
    return est


def training_set(n_gathers: int = 2000, crops: int = 8, n_its: int = 100, seed: int = TRAIN_SEED,
                 batch: int = 100):
    """(inputs, targets) of n_gathers * crops windows of 32 x 256: seeded
    128 x 512 gathers (gather_2d, seeds seed + i) blended in sum mode, read
    back at their shot times (the pseudo-deblended input), and deblended by
    the plain method on the GPU (n_its iterations, windows (32, 256)); both
    normalised by the input gather's RMS."""
    from . import deblend_batch

    rng = np.random.default_rng(seed)
    xs, ts = [], []
    for g0 in range(0, n_gathers, batch):
        gathers = [S.gather_2d(seed=seed + g, n_shots=128, nt=512, window=(32, 256),
                               n_its=n_its) for g in range(g0, min(n_gathers, g0 + batch))]
        outs = deblend_batch([dict(volumes=g.volumes, window_shapes=g.window_shapes,
                                   coords=g.coords, shottimes=g.shottimes, channels=g.channels,
                                   trace_types=g.trace_types, data=g.data) for g in gathers],
                             1.0, n_its)
        for g, o in zip(gathers, outs):
            x = g.data[0].astype(np.float32)
            y = np.asarray(o[0], np.float32)
            rms = float(np.sqrt(np.mean(x.astype(np.float64) ** 2))) or 1.0
            for _ in range(crops):
                i0 = int(rng.integers(0, x.shape[0] - 32 + 1))
                j0 = int(rng.integers(0, x.shape[1] - 256 + 1))
                xs.append(x[i0: i0 + 32, j0: j0 + 256] / rms)
                ts.append(y[i0: i0 + 32, j0: j0 + 256] / rms)
    return np.stack(xs), np.stack(ts)


def neighbour_lines(v, line_axis: int, nbr_axis: int, k: int):
    """Lines of the volume v along line_axis (the last axis is time) with
    their neighbours: [n][traces][time][2 k + 1], channel 0 the line itself,
    then the lines at offsets -1, +1, ..., -k, +k along nbr_axis (clamped at
    the edge) - the channel order agd_gpu_solve_learned feeds a network with
    2 k + 1 input channels."""
    v = np.asarray(v, np.float32)
    n_nb = v.shape[nbr_axis]
    chans = []
    for o in [0] + [s * m for m in range(1, k + 1) for s in (-1, 1)]:
        w = np.take(v, np.clip(np.arange(n_nb) + o, 0, n_nb - 1), axis=nbr_axis)
        a = np.moveaxis(w, line_axis, -2)
        chans.append(a.reshape(-1, a.shape[-2], a.shape[-1]))
    return np.stack(chans, -1)


def training_set_vibroseis(n_surveys: int = 40, crops: int = 1, n_its: int = 150,
                           seed: int = TRAIN_SEED, both_axes: bool = False,
                           neighbours: int = 0):
    """(inputs, targets) of 32 x 256 windows of receiver gathers from seeded
    small vibroseis surveys (vibroseis_4d with seeds seed + i: 16 sY x 32 sX
    x 16 channels x 2048 samples, the 256-sample 8-80 Hz sweep, windows
    (16, 16, 16, 256)) deblended by the plain method on the GPU; every line
    along sX (32 shots x 2048 samples) gives `crops` windows, normalised by
    the line's RMS; with both_axes also every line along sY (16 shots,
    zero-padded to 32 rows).  neighbours = k > 0: the surveys are 32 sY x
    16 sX instead, and the images are the lines along sY (the slow source
    axis, 32 shots) with the lines at sX offsets -1, +1, ..., -k, +k (the
    shots fired just before and after) as channels 1 .. 2 k: inputs
    [n][32][256][2 k + 1] (neighbour_lines), as agd_gpu_solve_learned feeds
    a multi-channel network."""
    from . import Problem

    if neighbours and both_axes:
        raise ValueError("neighbour channels are built for the lines along sY only")
    rng = np.random.default_rng(seed + 100000)
    xs, ts = [], []
    for i in range(n_surveys):
        n_sy, n_sx = (32, 16) if neighbours else (16, 32)
        sv = S.vibroseis_4d(seed=seed + i, n_sy=n_sy, n_sx=n_sx, n_ch=16, nt=2048,
                            window=(16, 16, 16, 256), n_its=n_its)
        p = Problem.from_survey(sv)
        out = p.solve(sv.data, 1.0, n_its)
        p.close()
        if neighbours:  # (sX, ch) lines along sY, neighbours along sX
            xc = neighbour_lines(sv.data[0], 0, 1, neighbours)
            y = neighbour_lines(out[0], 0, 1, 0)[..., 0]
            for xi, yi in zip(xc, y):
                rms = float(np.sqrt(np.mean(xi[..., 0].astype(np.float64) ** 2))) or 1.0
                for _ in range(crops):
                    j0 = int(rng.integers(0, 2048 - 256 + 1))
                    xs.append(xi[:, j0: j0 + 256] / rms)
                    ts.append(yi[:, j0: j0 + 256] / rms)
            continue
        x = np.moveaxis(sv.data[0], 1, 2).reshape(-1, 32, 2048)  # (sY, ch) lines along sX
        y = np.moveaxis(np.asarray(out[0], np.float32), 1, 2).reshape(-1, 32, 2048)
        if both_axes:  # (sX, ch) lines along sY, padded to 32 rows
            xs2 = np.moveaxis(sv.data[0], 0, 2).reshape(-1, 16, 2048)
            ys2 = np.moveaxis(np.asarray(out[0], np.float32), 0, 2).reshape(-1, 16, 2048)
            pad = ((0, 0), (0, 16), (0, 0))
            x = np.concatenate([x, np.pad(xs2, pad)])
            y = np.concatenate([y, np.pad(ys2, pad)])
        for xi, yi in zip(x, y):
            rms = float(np.sqrt(np.mean(xi.astype(np.float64) ** 2))) or 1.0
            for _ in range(crops):
                j0 = int(rng.integers(0, 2048 - 256 + 1))
                xs.append(xi[:, j0: j0 + 256] / rms)
                ts.append(yi[:, j0: j0 + 256] / rms)
    return np.stack(xs).astype(np.float32), np.stack(ts).astype(np.float32)


def train(family: str = "gather_2d", n: int = 2000, epochs: int = 8, batch: int = 32,
          lr: float | None = None, base_channels: int = 32, seed: int = 0,
          cosine: bool | None = None):
    """A network trained on the plain method's own results: family
    "gather_2d" (n receiver gathers, training_set, one input channel) or
    "vibroseis" (n small surveys, lines along sY with their two neighbours
    along sX as channels 1 and 2, training_set_vibroseis: on held-out
    surveys this warm-starts better than lines along sX, with or without
    neighbours along sY, and than the mean of both axes).  Adam; with cosine the learning
    rate of epoch e is lr (1 + cos(pi e / epochs)) / 2 (one agd_nn_train
    call per epoch, the optimiser state carried over).  Defaults, chosen on
    held-out surveys: lr 1e-3 with the cosine decay for "gather_2d", a
    constant 5e-4 for "vibroseis".
    Returns (net, per-epoch mean loss)."""
    if lr is None:
        lr = 5e-4 if family == "vibroseis" else 1e-3
    if cosine is None:
        cosine = family != "vibroseis"
    in_ch = 1
    if family == "vibroseis":
        x, t = training_set_vibroseis(n, neighbours=1)
        in_ch = 3
    else:
        x, t = training_set(n)
    net = WarmStartNet(base_channels, seed=seed, in_channels=in_ch)
    if not cosine:
        return net, net.train(x, t, batch=batch, epochs=epochs, lr=lr, seed=seed)
    losses = np.zeros(epochs)
    for e in range(epochs):
        rate = lr * 0.5 * (1.0 + np.cos(np.pi * e / epochs))
        losses[e] = net.train(x, t, batch=batch, epochs=1, lr=float(rate), seed=seed + e)[0]
    return net, losses


def _bind_warm(lib, dtype):
    if getattr(lib, "_agd_warm_bound", False):
        return
    rc = capi.real_ctype(dtype)
    rp = POINTER(rc)
    lib.agd_gpu_solve_warm.argtypes = [ctypes.c_void_p, rc, c_int, c_int, c_int, POINTER(rp),
                                       POINTER(rp)]
    lib.agd_gpu_solve_warm.restype = c_int
    lib.agd_gpu_warm_model.argtypes = [ctypes.c_void_p, POINTER(rp), rp]
    lib.agd_gpu_warm_model.restype = c_int
    lib._agd_warm_bound = True


def solve_warm(problem, data, estimate_patches, initial_factor: float, n_its: int,
               it_begin: int, print_freq: int = 0):
    """agd_gpu_solve_warm on a planned problem (agdeblend_b200.Problem):
    iterations [it_begin, n_its) of the plain schedule from the warm model
    of the estimate.  Returns the deblended patches."""
    lib = problem.lib
    _bind_warm(lib, problem.dtype)
    ptrs, keep = problem._data_ptrs(data, writable=True)
    eptrs, ekeep = problem._data_ptrs(estimate_patches)
    if lib.agd_gpu_solve_warm(problem.h, initial_factor, n_its, it_begin, print_freq, eptrs,
                              ptrs):
        raise RuntimeError("agd_gpu_solve_warm failed")
    return [k.reshape(s) for k, s in zip(keep, problem.shapes)]


def warm_model(problem, estimate_patches) -> np.ndarray:
    """The model (interleaved re, im) whose operator reproduces the estimate."""
    lib = problem.lib
    _bind_warm(lib, problem.dtype)
    eptrs, ekeep = problem._data_ptrs(estimate_patches)
    out = np.zeros(2 * problem.model_size, problem.dtype)
    if lib.agd_gpu_warm_model(problem.h, eptrs, out.ctypes.data_as(problem._rp)):
        raise RuntimeError("agd_gpu_warm_model failed")
    return out


def solve_learned(problem, net: WarmStartNet, data, initial_factor: float, n_its: int,
                  it_begin: int, print_freq: int = 0, overwrite_input: bool = False):
    """agd_gpu_solve_learned: the network's estimate of the deblended data
    (computed on the device from the uploaded input) as the warm start,
    then iterations [it_begin, n_its) of the plain schedule.  The input is
    left intact unless overwrite_input (as Problem.solve)."""
    lib = problem.lib
    _bind_warm(lib, problem.dtype)
    if not getattr(lib, "_agd_learned_bound", False):
        rc = capi.real_ctype(problem.dtype)
        lib.agd_gpu_solve_learned.argtypes = [ctypes.c_void_p, ctypes.c_void_p, rc, c_int, c_int,
                                              c_int, POINTER(POINTER(rc))]
        lib.agd_gpu_solve_learned.restype = c_int
        lib._agd_learned_bound = True
    ptrs, keep = problem._data_ptrs(data, writable=True, in_place=overwrite_input)
    if lib.agd_gpu_solve_learned(problem.h, net.h, initial_factor, n_its, it_begin, print_freq,
                                 ptrs):
        raise RuntimeError("agd_gpu_solve_learned failed")
    return [k.reshape(s) for k, s in zip(keep, problem.shapes)]
