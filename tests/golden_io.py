"""Loads the golden fixtures written by tests/golden/make_golden.py."""
import os

import numpy as np

from agdeblend_b200.synthetic import Survey

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
OPS_CASES = ["gather_2d", "two_volume_3d", "wavelet_4d", "random_neighbours"]


def load_ops(name):
    z = np.load(os.path.join(GOLDEN, f"ops_{name}.npz"))
    n_p = int(z["n_patches"])
    n_v = int(z["n_volumes"])

    def seq(prefix, n):
        return [z[f"{prefix}_{i}"] for i in range(n)]

    wl = widx = wv = None
    if bool(z["has_wavelets"]):
        wl = [int(v) for v in z["wavelet_lengths"]]
        widx = seq("wavelet_idxs", n_p)
        wv = seq("wavelet", len(wl))
    sv = Survey(name, [int(v) for v in z["volumes"]], [int(v) for v in z["n_dims"]],
                [list(map(int, w)) for w in seq("window_shape", n_v)],
                [list(map(int, c)) for c in seq("coords", n_p)],
                [list(map(int, s)) for s in seq("shape", n_p)], seq("shottimes", n_p),
                seq("channels", n_p), seq("trace_types", n_p), seq("data", n_p),
                seq("data", n_p), 10, wavelet_lengths=wl, wavelet_idxs=widx, wavelets=wv)
    ref = dict(record_in=z["record_in"], model_adjoint=z["model_adjoint"],
               record_forward=z["record_forward"], blend_input=z["blend_input"],
               stepsize=float(z["stepsize"]), output=seq("output", n_p))
    return sv, ref


def sketch(arrays, k: int = 64, chunk: int = 1 << 20) -> np.ndarray:
    """k random +-1 projections of the concatenated arrays (float64).  The
    signs come from a fixed integer hash of (element index, projection), so
    they need no random generator and are identical on every machine.  For
    any x, E |sketch(x)|^2 / k = |x|^2, so |sketch(a) - sketch(b)| /
    |sketch(b)| estimates the relative L2 difference (to about 1/sqrt(k/2))."""
    flat = np.concatenate([np.asarray(a, np.float64).reshape(-1) for a in arrays])
    out = np.zeros(k)
    mult = np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):  # the hash wraps modulo 2^64 on purpose
        for s0 in range(0, flat.size, chunk):
            x = flat[s0: s0 + chunk]
            idx = np.arange(s0, s0 + x.size, dtype=np.uint64)
            for j in range(k):
                h = (idx + np.uint64(j) * np.uint64(0x632BE59BD9B4E019)) * mult
                sign = 1.0 - 2.0 * ((h >> np.uint64(63)).astype(np.float64))
                out[j] += float(np.dot(sign, x))
    return out
