"""Oracle (test infrastructure only): a float64 numpy restatement of the
reference's deblending path, used to check the CUDA implementation.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import this module.  The product never calls it.

It restates, function by function, what the reference computes (file:line
into the reference project):

planning
  * ``_n_model_times``          src/model.c:326-357 (set_n_model_times)
  * ``_add_interval``           src/blend.c:49-151 (interval merge, quirks kept)
  * ``_blend_config``           src/blend.c:176-342,585-691
  * ``_blend_coords``           src/blend.c:693-760
  * ``_patch_use_taper``        src/model.c:20-50,149-188
  * ``_space_windows``          src/model.c:456-745
  * ``_taper``                  src/fk.c:28-73
  * ``_fk_window``              src/fk.c:75-169
  * ``_wavelet_spectrum``       src/wavelet.c:188-237
operators
  * ``fk_forward``              src/fk.c:307-373
  * ``fk_adjoint``              src/fk.c:375-452
  * ``wavelet_operator``        src/wavelet.c:239-301
  * ``blend_sum`` / ``blend_adjoint`` / ``blend_mean``  src/blend.c:936-1292
  * ``forward`` (model_forward) src/model.c:1067-1114
  * ``adjoint`` (model_adjoint_update) src/model.c:1116-1157
  * ``stepsize``                src/model.c:1230-1312
  * ``blend_input``             src/blend.c:1294-1335
  * ``threshold``               src/model.c:1392-1423
  * ``set_output``              src/model.c:1425-1515
drivers
  * ``lambda_schedule``         src/agdeblend.c:526-533,623-627
  * ``deblend`` (agd_deblend)   src/agdeblend.c:511-649
  * ``blend`` (agd_blend)       src/agdeblend.c:800-938

FFTs use numpy's pocketfft in float64 with the unnormalised FFTW conventions
(``irfftn`` scaled by the transform size).
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
from dataclasses import dataclass, field

import numpy as np

LIVE, BAD, MISSING = 0, 1, 2
BLEND_SUM, BLEND_MEAN, BLEND_OVERWRITE = 0, 1, 2
PAD_FRACTION = 0.25
TARGET_LAMB = 1e-3

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
for _fn in ("expf", "logf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]
_libm.powf.restype = ctypes.c_float
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]


class OracleError(RuntimeError):
    pass


# ----------------------------------------------------------------- planning


def _n_model_times(nt: int, lt: int, wl: int) -> tuple[int, int]:
    """(n_times_fk, n_times_conv) for one patch (src/model.c:336-351)."""
    h = lt // 2
    n_before = nt - wl + 1
    n_win = (n_before + h - 1) // h + 1
    n_fk = (n_win + 1) * h
    return n_fk, n_fk + wl - 1


def _overlaps(a, b) -> bool:
    return a[0] < b[1] and a[1] > b[0]


def _adjacent(a, b) -> bool:
    return a[0] == b[1] or a[1] == b[0]


def _add_interval(ivs: list, new: tuple) -> None:
    """Merge ``new`` into the channel's interval list, keeping the reference's
    search order: later matches are tested against the new interval (not the
    grown one) and the scan resumes one past a deleted entry
    (src/blend.c:113-151)."""

    def find(start):
        for i in range(start, len(ivs)):
            if _overlaps(new, ivs[i]) or _adjacent(new, ivs[i]):
                return i
        return -1

    first = find(0)
    if first < 0:
        ivs.append([new[0], new[1]])
        return
    ivs[first][0] = min(ivs[first][0], new[0])
    ivs[first][1] = max(ivs[first][1], new[1])
    start = first + 1
    while True:
        i = find(start)
        if i < 0:
            break
        ivs[first][0] = min(ivs[first][0], ivs[i][0])
        ivs[first][1] = max(ivs[first][1], ivs[i][1])
        del ivs[i]
        start = i + 1


@dataclass
class BlendConfig:
    channel_values: list
    intervals: list  # per channel: list of [start, stop]
    seg_offset: dict  # (ch, iv) -> flat offset
    total: int
    mute: list  # (flat offset, n)

    def channel_index(self, value: int, ttype: int) -> int:
        if ttype == MISSING:
            return -1
        try:
            return self._lookup[value]
        except KeyError:
            return -1

    def __post_init__(self):
        self._lookup = {v: i for i, v in enumerate(self.channel_values)}


def _blend_config(shottimes, n_times, channels, trace_types) -> BlendConfig:
    """set_blend_config (src/blend.c:629-691) on per-patch trace lists."""
    values: list = []
    seen: dict = {}
    for ch_p, tt_p in zip(channels, trace_types):
        for c, t in zip(ch_p.tolist(), tt_p.tolist()):
            if t == MISSING:
                continue
            if c not in seen:
                seen[c] = len(values)
                values.append(c)
    intervals = [[] for _ in values]
    mutes = [[] for _ in values]
    for st_p, nt, ch_p, tt_p in zip(shottimes, n_times, channels, trace_types):
        for s, c, t in zip(st_p.tolist(), ch_p.tolist(), tt_p.tolist()):
            if t == MISSING:
                continue
            ci = seen[c]
            _add_interval(intervals[ci], (s, s + nt))
            if t == BAD:
                _add_interval(mutes[ci], (s, s + nt))
    seg_offset = {}
    off = 0
    for ci, ivs in enumerate(intervals):
        for ii, iv in enumerate(ivs):
            seg_offset[(ci, ii)] = off
            off += iv[1] - iv[0]
    mute = []
    for ci in range(len(values)):
        for m in mutes[ci]:
            for ii, iv in enumerate(intervals[ci]):
                if _overlaps(m, iv):
                    a = max(m[0], iv[0])
                    b = min(m[1], iv[1])
                    mute.append((seg_offset[(ci, ii)] + a - iv[0], b - a))
    return BlendConfig(values, intervals, seg_offset, off, mute)


def _blend_coords(cfg: BlendConfig, shottimes, n_times, channels, trace_types):
    """Per trace (flat record start, trace_start, n) or None
    (set_blend_coords, src/blend.c:693-726)."""
    out = []
    for s, c, t in zip(shottimes.tolist(), channels.tolist(), trace_types.tolist()):
        ci = cfg.channel_index(c, t)
        coord = None
        if t != MISSING and ci >= 0:
            for ii, iv in enumerate(cfg.intervals[ci]):
                if _overlaps((s, s + n_times), iv):
                    a = max(s, iv[0])
                    b = min(s + n_times, iv[1])
                    coord = (cfg.seg_offset[(ci, ii)] + a - iv[0], a - s, b - a)
                    break
        out.append(coord)
    return out


def _patch_use_taper(volumes, n_dims, coords):
    """use_taper per patch: 1 on an edge that touches another patch of the
    same volume, diagonals included (src/model.c:20-50,149-188)."""
    res = []
    for p, (vol, cp) in enumerate(zip(volumes, coords)):
        nd = n_dims[vol] - 1
        ut = [0] * (2 * nd)
        for q, (vol2, cq) in enumerate(zip(volumes, coords)):
            if q == p or vol2 != vol:
                continue
            if any(cq[d] not in (cp[d] - 1, cp[d], cp[d] + 1) for d in range(nd)):
                continue
            for d in range(nd):
                if cq[d] == cp[d] - 1:
                    ut[2 * d] = 1
                elif cq[d] == cp[d] + 1:
                    ut[2 * d + 1] = 1
        res.append(ut)
    return res


def _taper(length: int, left: int, right: int) -> np.ndarray:
    """Hann taper of half the window length on the requested sides
    (src/fk.c:28-73)."""
    tl = length // 2
    w = np.ones(length)
    if tl > 0:
        i = np.arange(tl)
        if left:
            w[:tl] = 0.5 * (1 - np.cos(2 * np.pi * i / (2 * tl)))
        if right:
            w[length - tl:] = 0.5 * (1 - np.cos(2 * np.pi * (tl + i) / (2 * tl)))
    return w


@dataclass
class Window:
    patch: int
    coords: list
    shape: list  # space shape
    use_taper: list  # 2 per space dim
    trace_index: np.ndarray  # patch trace index of each window trace
    lt: int = 0
    n_tw: int = 0
    padded: list = field(default_factory=list)  # space..., time
    scaler: float = 0.0
    tapers: list = field(default_factory=list)  # space..., time
    n_fk: int = 0
    conv: int = 0
    blend: list = field(default_factory=list)
    wavelet_src: list | None = None  # per trace: source config index or -1

    @property
    def n_freq(self) -> int:
        return self.padded[-1] // 2 + 1

    @property
    def model_shape(self) -> tuple:
        return (self.n_tw, *self.padded[:-1], self.n_freq)

    @property
    def n_traces(self) -> int:
        return int(np.prod(self.shape)) if self.shape else 1

    def space_taper(self) -> np.ndarray:
        t = np.ones(())
        for d in range(len(self.shape)):
            t = np.multiply.outer(t, self.tapers[d])
        return t.reshape(-1)


def _space_windows(volumes, n_dims, window_shapes, coords, shapes, patch_ut):
    """Windows in the reference's order (src/model.c:470-745)."""
    wins = []
    for p, vol in enumerate(volumes):
        nd = n_dims[vol] - 1
        pshape = shapes[p]
        wshape = window_shapes[vol]
        per_dim = []
        for d in range(nd):
            n, L = pshape[d], wshape[d]
            nw = 1 if L == n else n // (L // 2) - 1
            tl = L // 2
            base = (n - tl) // nw + tl
            n_larger = n - tl - (base - tl) * nw
            starts, lens = [], []
            start = 0
            for i in range(nw):
                ln = base + (1 if i < n_larger else 0)
                starts.append(start)
                lens.append(ln)
                start += ln - tl
            per_dim.append((starts, lens, nw))
        for idx in np.ndindex(*[pd[2] for pd in per_dim]):
            wc = [per_dim[d][0][idx[d]] for d in range(nd)]
            ws = [per_dim[d][1][idx[d]] for d in range(nd)]
            ut = []
            for d in range(nd):
                ut.append(patch_ut[p][2 * d] if idx[d] == 0 else 1)
                ut.append(patch_ut[p][2 * d + 1] if idx[d] == per_dim[d][2] - 1 else 1)
            grids = np.meshgrid(*[np.arange(wc[d], wc[d] + ws[d]) for d in range(nd)], indexing="ij")
            tidx = np.ravel_multi_index([g.reshape(-1) for g in grids], tuple(pshape[:nd]))
            wins.append(Window(p, wc, ws, ut, tidx))
    return wins


def _fk_window(win: Window, n_fk: int, conv: int, lt: int) -> None:
    """set_fk_window_config (src/fk.c:75-169)."""
    full = list(win.shape) + [lt]
    win.lt = lt
    win.n_tw = n_fk // (lt // 2) - 1
    win.padded = [int(math.ceil(L * (1 + PAD_FRACTION))) for L in full]
    win.scaler = 1.0 / math.sqrt(float(np.prod(win.padded)))
    ut = list(win.use_taper) + [1, 1]
    win.tapers = [_taper(full[d], ut[2 * d], ut[2 * d + 1]) for d in range(len(full))]
    win.n_fk = n_fk
    win.conv = conv


def _wavelet_spectrum(wavelet: np.ndarray, n: int) -> np.ndarray:
    """Phase-only spectrum scaled by 1/n (src/wavelet.c:188-237)."""
    buf = np.zeros(n)
    buf[: len(wavelet)] = wavelet
    ang = np.angle(np.fft.rfft(buf))
    return np.exp(1j * ang) / n


@dataclass
class Plan:
    """Everything set_model (src/model.c:932-1065) prepares, plus the
    step size (src/model.c:1230-1312)."""

    n_patches: int
    volumes: list
    n_dims: list
    shapes: list
    shottimes: list
    channels: list
    trace_types: list
    n_fk: list
    conv: list
    cfg: BlendConfig
    windows: list
    spectra: list  # per wavelet source config
    step: float = 0.0

    @property
    def model_sizes(self):
        return [int(np.prod(w.model_shape)) for w in self.windows]

    def zero_model(self):
        return [np.zeros(w.model_shape, complex) for w in self.windows]


def _volume_wavelet_lengths(volumes, n_traces, trace_types, wavelet_lengths, wavelet_idxs):
    """set_volume_wavelet_lengths (src/utils.c:72-123)."""
    nv = max(volumes) + 1
    out = [0] * nv
    if wavelet_idxs is None:
        return [1] * nv
    for p, vol in enumerate(volumes):
        if out[vol] == 0:
            for t in range(n_traces[p]):
                if trace_types[p][t] == LIVE:
                    out[vol] = int(wavelet_lengths[int(wavelet_idxs[p][t])])
                    if out[vol] <= 0:
                        raise OracleError("Wavelet lengths must be positive")
                    break
    return [v if v else 1 for v in out]


def make_plan(volumes, n_dims, window_shapes, coords, shapes, shottimes, channels,
              trace_types, wavelet_lengths=None, wavelet_idxs=None, wavelets=None) -> Plan:
    volumes = [int(v) for v in volumes]
    n_dims = [int(v) for v in n_dims]
    shapes = [tuple(int(s) for s in sh) for sh in shapes]
    n_patches = len(volumes)
    shottimes = [np.asarray(s, np.int64).reshape(-1) for s in shottimes]
    channels = [np.asarray(c, np.int64).reshape(-1) for c in channels]
    trace_types = [np.asarray(t, np.int64).reshape(-1) for t in trace_types]
    n_traces = [int(np.prod(sh[:-1])) for sh in shapes]
    nts = [sh[-1] for sh in shapes]
    lts = [int(window_shapes[v][n_dims[v] - 1]) for v in volumes]
    wl_vol = _volume_wavelet_lengths(volumes, n_traces, trace_types, wavelet_lengths,
                                     wavelet_idxs)
    n_fk, conv = [], []
    for p in range(n_patches):
        a, b = _n_model_times(nts[p], lts[p], wl_vol[volumes[p]])
        n_fk.append(a)
        conv.append(b)
    shifted = [shottimes[p] - lts[p] // 2 for p in range(n_patches)]
    cfg = _blend_config(shifted, conv, channels, trace_types)
    put = _patch_use_taper(volumes, n_dims, coords)
    for p, vol in enumerate(volumes):
        for d in range(n_dims[vol] - 1):
            if (put[p][2 * d] or put[p][2 * d + 1]) and window_shapes[vol][d] % 2 == 1:
                raise OracleError("window shapes may only be odd if there is no tapering")
    wins = _space_windows(volumes, n_dims, window_shapes, coords, shapes, put)
    kept = []
    src_keys: list = []
    spectra: list = []
    for w in wins:
        p = w.patch
        tt = trace_types[p][w.trace_index]
        if not np.any(tt == LIVE):
            continue
        _fk_window(w, n_fk[p], conv[p], lts[p])
        if wavelet_idxs is not None:
            widx = np.asarray(wavelet_idxs[p]).reshape(-1)[w.trace_index]
            src = []
            for t, wi in zip(tt.tolist(), widx.tolist()):
                if t != LIVE:
                    src.append(-1)
                    continue
                key = (int(wi), conv[p])
                if key not in src_keys:
                    src_keys.append(key)
                    spectra.append(_wavelet_spectrum(np.asarray(wavelets[key[0]], float)[
                        : int(wavelet_lengths[key[0]])], key[1]))
                src.append(src_keys.index(key))
            w.wavelet_src = src
        w.blend = _blend_coords(cfg, shifted[p][w.trace_index], conv[p],
                                channels[p][w.trace_index], tt)
        kept.append(w)
    plan = Plan(n_patches, volumes, n_dims, shapes, shottimes, channels, trace_types,
                n_fk, conv, cfg, kept, spectra)
    plan.step = stepsize(plan)
    return plan


# ---------------------------------------------------------------- operators


def fk_forward(w: Window, x: np.ndarray) -> np.ndarray:
    """[T][P..][F] complex -> [n_traces][conv] real (src/fk.c:307-373)."""
    nd = len(w.shape)
    axes = tuple(range(1, nd + 2))
    u = np.fft.irfftn(x, s=w.padded, axes=axes) * float(np.prod(w.padded))
    u = u[(slice(None),) + tuple(slice(0, L) for L in w.shape) + (slice(0, w.lt),)]
    u = u.reshape(w.n_tw, w.n_traces, w.lt) * (w.scaler * w.space_taper())[None, :, None]
    u = u * w.tapers[-1][None, None, :]
    h = w.lt // 2
    y = np.zeros((w.n_traces, w.conv))
    for t in range(w.n_tw):
        y[:, t * h: t * h + w.lt] += u[t]
    return y


def fk_adjoint(w: Window, y: np.ndarray) -> np.ndarray:
    """[n_traces][conv] real -> [T][P..][F] complex (src/fk.c:375-452)."""
    nd = len(w.shape)
    h = w.lt // 2
    seg = np.stack([y[:, t * h: t * h + w.lt] for t in range(w.n_tw)])
    seg = seg * (w.scaler * w.space_taper())[None, :, None] * w.tapers[-1][None, None, :]
    u = np.zeros((w.n_tw, *w.padded))
    u[(slice(None),) + tuple(slice(0, L) for L in w.shape) + (slice(0, w.lt),)] = seg.reshape(
        w.n_tw, *w.shape, w.lt)
    x = np.fft.rfftn(u, axes=tuple(range(1, nd + 2)))
    pt = w.padded[-1]
    x[..., 1: 1 + (pt - 1) // 2] *= 2
    return x


def wavelet_operator(plan: Plan, w: Window, y: np.ndarray, direction: int) -> np.ndarray:
    """Phase-only wavelet convolution (+1) / correlation (-1) per trace
    (src/wavelet.c:239-301); non-live traces only round-trip the unnormalised
    transform pair, i.e. are scaled by the transform length."""
    if w.wavelet_src is None:
        return y
    src = np.asarray(w.wavelet_src)
    if not np.any(src >= 0):
        return y
    n = w.conv
    Y = np.fft.rfft(y, axis=1)
    for i, s in enumerate(src.tolist()):
        if s >= 0:
            sp = plan.spectra[s]
            Y[i] *= sp if direction > 0 else np.conj(sp)
    return np.fft.irfft(Y, n, axis=1) * n


def blend_sum(coords, y: np.ndarray, rec: np.ndarray) -> None:
    """rec += B y (src/blend.c:936-960)."""
    for i, c in enumerate(coords):
        if c is not None:
            off, ts, n = c
            rec[off: off + n] += y[i, ts: ts + n]


def blend_adjoint(coords, rec: np.ndarray, length: int) -> np.ndarray:
    """B^H: gather record segments into traces (src/blend.c:1262-1292)."""
    y = np.zeros((len(coords), length))
    for i, c in enumerate(coords):
        if c is not None:
            off, ts, n = c
            y[i, ts: ts + n] = rec[off: off + n]
    return y


def apply_mute(cfg: BlendConfig, rec: np.ndarray) -> None:
    for off, n in cfg.mute:
        rec[off: off + n] = 0.0


def forward(plan: Plan, x: list) -> np.ndarray:
    """model_forward: mute(sum_w B_w W_w F_w x_w) (src/model.c:1067-1114)."""
    rec = np.zeros(plan.cfg.total)
    for w, xw in zip(plan.windows, x):
        y = wavelet_operator(plan, w, fk_forward(w, xw), +1)
        blend_sum(w.blend, y, rec)
    apply_mute(plan.cfg, rec)
    return rec


def adjoint(plan: Plan, rec: np.ndarray) -> list:
    """A^H r per window (model_adjoint_update with stepsize -1 on a zero
    model, src/model.c:1116-1157)."""
    out = []
    for w in plan.windows:
        y = blend_adjoint(w.blend, rec, w.conv)
        y = wavelet_operator(plan, w, y, -1)
        out.append(fk_adjoint(w, y))
    return out


def stepsize(plan: Plan) -> float:
    """0.5 / max(1, max blend-sum of the space tapers) (src/model.c:1230-1312)."""
    rec = np.zeros(plan.cfg.total)
    for w in plan.windows:
        y = np.repeat(w.space_taper()[:, None], w.conv, axis=1)
        blend_sum(w.blend, y, rec)
    factor = max(1.0, float(rec.max()) if rec.size else 1.0)
    return 0.5 / factor


def blend_mean(cfg: BlendConfig, coords_per_patch, data, taper_length: int) -> np.ndarray:
    """Mean blend with optional cosine edge weights (src/blend.c:1155-1260)."""
    rec = np.zeros(cfg.total)
    cnt = np.zeros(cfg.total)
    taper = None
    if taper_length > 1:
        i = np.arange(taper_length)
        taper = np.cos(0.5 * np.pi * (taper_length - i) / (taper_length + 1))
    for coords, d in zip(coords_per_patch, data):
        for i, c in enumerate(coords):
            if c is None:
                continue
            off, ts, n = c
            wgt = np.ones(n)
            if taper is not None:
                t = np.arange(n)
                edge = np.minimum(t, n - 1 - t)
                sel = edge < taper_length
                wgt[sel] = taper[edge[sel]]
            rec[off: off + n] += d[i, ts: ts + n] * wgt
            cnt[off: off + n] += wgt
    pos = cnt > 0
    rec[pos] /= cnt[pos]
    return rec


def blend_input(plan: Plan, data: list) -> np.ndarray:
    """d = mute(mean blend of the input at the raw shot times) on the blend
    config of the model (src/blend.c:1294-1335)."""
    coords = [_blend_coords(plan.cfg, plan.shottimes[p], plan.shapes[p][-1],
                            plan.channels[p], plan.trace_types[p])
              for p in range(plan.n_patches)]
    flat = [np.asarray(d, float).reshape(-1, plan.shapes[p][-1]) for p, d in enumerate(data)]
    rec = blend_mean(plan.cfg, coords, flat, 0)
    apply_mute(plan.cfg, rec)
    return rec


def threshold(x: list, lamb: float) -> list:
    """Complex soft threshold (src/model.c:1392-1423)."""
    out = []
    for xw in x:
        a2 = xw.real ** 2 + xw.imag ** 2
        keep = a2 > lamb * lamb
        a = np.sqrt(np.where(keep, a2, 1.0))
        out.append(np.where(keep, xw * ((a - lamb) / a), 0.0))
    return out


def set_output(plan: Plan, x: list) -> list:
    """Window sum of W F x into the patches (src/model.c:1425-1515)."""
    data = [np.zeros((int(np.prod(sh[:-1])), sh[-1])) for sh in plan.shapes]
    for w, xw in zip(plan.windows, x):
        y = wavelet_operator(plan, w, fk_forward(w, xw), +1)
        nt = plan.shapes[w.patch][-1]
        h = w.lt // 2
        np.add.at(data[w.patch], w.trace_index, y[:, h: h + nt])
    return [d.reshape(plan.shapes[p]) for p, d in enumerate(data)]


def lambda_schedule(initial_factor: float, n_its: int, double: bool = False):
    """(decay, first_linear_it, linear_slope / lambda_0) evaluated as the
    reference does (src/agdeblend.c:526-533): in single precision with the C
    library's expf/logf/powf for the float build, in double precision for the
    double build."""
    if double:
        decay = math.exp(math.log(TARGET_LAMB / initial_factor) / n_its)
        ld = math.log(decay)
        fli = int((ld * (n_its - 1.0) + 1.0) / ld)
        slope = initial_factor * decay ** fli / (n_its - 1 - fli)
        return decay, fli, slope
    f32 = np.float32
    f = f32(initial_factor)
    decay = _libm.expf(f32(_libm.logf(f32(f32(TARGET_LAMB) / f)) / f32(n_its)))
    decay = f32(decay)
    ld = f32(_libm.logf(decay))
    fli = int(f32(f32(ld * f32(f32(n_its) - f32(1.0)) + f32(1.0)) / ld))
    slope = f32(f * f32(_libm.powf(decay, f32(fli))) / f32(n_its - 1 - fli))
    return float(decay), fli, float(slope)


def lambdas(lamb0: float, initial_factor: float, n_its: int, double: bool = False) -> list:
    """Threshold used after the initial step and after each iteration."""
    decay, fli, slope = lambda_schedule(initial_factor, n_its, double)
    slope *= lamb0
    lamb = lamb0 * initial_factor
    out = [lamb]
    for it in range(1, n_its):
        if it < fli:
            lamb *= decay
        else:
            lamb = (n_its - 1 - it) * slope
        out.append(lamb)
    return out


def deblend(plan: Plan, data: list, initial_factor: float, n_its: int,
            callback=None, double_schedule: bool = False) -> list:
    """agd_deblend's solver (src/agdeblend.c:584-633) in float64; the
    threshold schedule follows the float (default) or the double build."""
    d = blend_input(plan, data)
    step = plan.step
    x = [-step * g for g in adjoint(plan, d)]
    lamb0 = math.sqrt(max(float(np.max(xw.real ** 2 + xw.imag ** 2)) if xw.size else 0.0
                          for xw in x))
    lams = lambdas(lamb0, initial_factor, n_its, double_schedule)
    x = threshold(x, lams[0])
    for it in range(1, n_its):
        r = forward(plan, x) - d
        if callback is not None:
            callback(it, float(np.sqrt(np.sum(r * r))))
        g = adjoint(plan, r)
        x = [xw - step * gw for xw, gw in zip(x, g)]
        x = threshold(x, lams[it])
    return set_output(plan, x)


def blend(n_times, shottimes, channels, trace_types, data, blend_mode, taper_length,
          n_times_out, shottimes_out, channels_out, trace_types_out) -> list:
    """agd_blend (src/agdeblend.c:800-938) on per-patch trace arrays."""
    st = [np.asarray(s, np.int64).reshape(-1) for s in shottimes]
    ch = [np.asarray(c, np.int64).reshape(-1) for c in channels]
    tt = [np.asarray(t, np.int64).reshape(-1) for t in trace_types]
    cfg = _blend_config(st, list(n_times), ch, tt)
    coords = [_blend_coords(cfg, st[p], n_times[p], ch[p], tt[p]) for p in range(len(st))]
    flat = [np.asarray(d, float).reshape(-1, n_times[p]) for p, d in enumerate(data)]
    if blend_mode == BLEND_MEAN:
        rec = blend_mean(cfg, coords, flat, taper_length)
    else:
        rec = np.zeros(cfg.total)
        for cs, d in zip(coords, flat):
            for i, c in enumerate(cs):
                if c is None:
                    continue
                off, ts, n = c
                if blend_mode == BLEND_SUM:
                    rec[off: off + n] += d[i, ts: ts + n]
                else:
                    rec[off: off + n] = d[i, ts: ts + n]
    apply_mute(cfg, rec)
    out = []
    for p in range(len(shottimes_out)):
        so = np.asarray(shottimes_out[p], np.int64).reshape(-1)
        co = np.asarray(channels_out[p], np.int64).reshape(-1)
        to = np.asarray(trace_types_out[p], np.int64).reshape(-1)
        cs = _blend_coords(cfg, so, n_times_out[p], co, to)
        out.append(blend_adjoint(cs, rec, n_times_out[p]))
    return out


# ------------------------------------------------------- layout conversions


def model_to_flat(x: list) -> np.ndarray:
    """Concatenate windows in the reference's model layout (interleaved)."""
    if not x:
        return np.zeros(0)
    return np.concatenate([xw.reshape(-1) for xw in x])


def flat_to_model(plan: Plan, flat: np.ndarray) -> list:
    out = []
    off = 0
    for w in plan.windows:
        n = int(np.prod(w.model_shape))
        out.append(np.asarray(flat[off: off + n]).reshape(w.model_shape))
        off += n
    return out
