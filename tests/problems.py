"""Random deblending problems in the style of the reference's own tests
(src/model_test.cpp:598-700 and src/test.cpp:432-561): 1-3 patches of 2-4
dimensions, small random shapes and windows, random shot times, channels and
trace types, optional wavelets, and optionally neighbouring patches of one
volume so that patch-edge tapers are exercised."""
from __future__ import annotations

import numpy as np

from agdeblend_b200.synthetic import BAD, LIVE, MISSING, Survey


def random_problem(seed: int, wavelets: bool = False, neighbours: bool = False,
                   bad_missing: bool = True, max_dims: int = 4) -> Survey:
    rng = np.random.default_rng(seed)
    n_patches = int(rng.integers(1, 4))
    n_dims_p = [int(rng.integers(2, max_dims + 1)) for _ in range(n_patches)]
    if neighbours:
        n_patches = 2
        nd = int(rng.integers(2, max_dims + 1))
        n_dims_p = [nd, nd]
    shapes, windows, coords = [], [], []
    for p in range(n_patches):
        nd = n_dims_p[p]
        sh, wn = [], []
        for d in range(nd):
            s = int(rng.integers(8, 17))
            w = int(rng.integers(8, s + 1))
            if w != s or d == nd - 1:
                w = max(4, (w // 4) * 4)
            sh.append(s)
            wn.append(w)
        shapes.append(sh)
        windows.append(wn)
        coords.append([0] * (nd - 1))
    if neighbours:
        windows[1] = list(windows[0])
        shapes[1] = [max(s, w) for s, w in zip(shapes[1], windows[1])]
        shapes[1][-1] = shapes[0][-1]
        for d in range(n_dims_p[0] - 1):  # neighbours must have even windows
            for p in (0, 1):
                if windows[p][d] % 2:
                    windows[p][d] -= 1
        coords[1][int(rng.integers(0, n_dims_p[0] - 1))] = 1
        volumes = [0, 0]
        window_shapes = [windows[0]]
        n_dims = [n_dims_p[0]]
    else:
        volumes = list(range(n_patches))
        window_shapes = windows
        n_dims = n_dims_p
    n_traces = [int(np.prod(s[:-1])) for s in shapes]
    total = sum(n * s[-1] for n, s in zip(n_traces, shapes))
    st_max = max(total // 3, 1)
    ch_max = 1 + sum(n_traces) // 10
    shottimes, channels, ttypes, data = [], [], [], []
    for p in range(n_patches):
        shottimes.append(rng.integers(0, st_max, n_traces[p]).astype(np.int64))
        channels.append(rng.integers(0, ch_max, n_traces[p]).astype(np.int32))
        if bad_missing:
            tt = rng.choice([LIVE, LIVE, LIVE, LIVE, BAD, MISSING], n_traces[p]).astype(np.int32)
        else:
            tt = np.zeros(n_traces[p], np.int32)
        tt[0] = LIVE
        ttypes.append(tt)
        data.append(rng.uniform(-0.5, 0.5, shapes[p]).astype(np.float32))
    wl = widx = wv = None
    if wavelets:
        n_w = int(rng.integers(1, 3))
        lens = {}
        wl, widx = [], []
        vol_len = {v: int(rng.integers(1, 6)) for v in set(volumes)}
        wv = []
        # one wavelet per volume length keeps "same length within a volume"
        per_vol = {}
        for v in sorted(set(volumes)):
            per_vol[v] = len(wl)
            for _ in range(n_w):
                wl.append(vol_len[v])
                wv.append(rng.uniform(-1, 1, vol_len[v]).astype(np.float32))
        for p in range(n_patches):
            widx.append((per_vol[volumes[p]] + rng.integers(0, n_w, n_traces[p])).astype(np.int32))
        del lens
    return Survey(f"random_{seed}", volumes, n_dims, window_shapes, coords, shapes, shottimes,
                  channels, ttypes, data, [d.copy() for d in data], 20,
                  wavelet_lengths=wl, wavelet_idxs=widx, wavelets=wv)
