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
