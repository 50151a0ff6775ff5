"""Seeded synthetic surveys with the shapes of the benchmark workloads.

The reference measures on seeded synthetic gathers only (examples/make_data.c);
no public dataset is involved.  Each generator returns the arguments of
``agd_deblend`` (per-patch arrays) plus the unblended truth, with
time in samples at dt = 4 ms.

Workloads (sizes as named in the benchmark specification):
  * ``gather_2d``      128 shots x 512 samples, one channel, window (32, 256)
  * ``two_volume_3d``  2 source volumes of (64 channels x 128 shots x 1024),
                       interleaved jittered shot times, 4 % bad and 4 % missing
                       traces, two 3 s gaps in the records, window (16, 32, 256)
  * ``vibroseis_4d``   (sY, sX, channel, time) = (32, 64, 32, 2048) convolved
                       with a 256-sample 8-80 Hz sweep, window (16, 16, 16, 256)
  * ``uneven_gathers`` many 2-D gathers of random size and window

The blended input is the record of summed overlapping traces read back at
each trace's shot time, i.e. ``agd_blend`` in sum mode with the same input
and output geometry (src/agdeblend.c:800-938 of the reference); bad traces'
spans are zeroed in the record, missing traces contribute nothing and read
back as zeros.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

LIVE, BAD, MISSING = 0, 1, 2
DT = 0.004
SAMPLES_PER_S = 250


@dataclass
class Survey:
    """Arguments of one agd_deblend call plus the unblended truth."""

    name: str
    volumes: list
    n_dims: list
    window_shapes: list
    coords: list
    shapes: list
    shottimes: list  # per patch, int64 [n_traces]
    channels: list  # per patch, int32 [n_traces]
    trace_types: list  # per patch, int32 [n_traces]
    data: list  # per patch, float32 [space..., time] (blended input)
    truth: list  # per patch, float32 [space..., time]
    n_its: int
    initial_factor: float = 1.0
    wavelet_lengths: list | None = None
    wavelet_idxs: list | None = None
    wavelets: list | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n_patches(self) -> int:
        return len(self.volumes)

    def n_samples(self) -> int:
        return int(sum(d.size for d in self.data))


def _ricker(t: np.ndarray, f: float = 20.0) -> np.ndarray:
    a = (np.pi * f * t) ** 2
    return (1 - 2 * a) * np.exp(-a)


def _add_events(out: np.ndarray, times: np.ndarray, amps: np.ndarray,
                f: float = 20.0, half: int = 16) -> None:
    """Add a Ricker wavelet at fractional sample ``times[trace]`` with
    amplitude ``amps`` to each trace of ``out`` ([n_traces, nt])."""
    n_tr, nt = out.shape
    base = np.floor(times).astype(np.int64)
    rows = np.arange(n_tr)
    for k in range(-half, half + 1):
        idx = base + k
        ok = (idx >= 0) & (idx < nt)
        val = amps * _ricker((idx - times) * DT, f)
        np.add.at(out, (rows[ok], idx[ok]), val[ok])


def _events(rng, n_traces, offsets_m, nt, channel_shift=None, n_lin=6, n_hyp=6):
    """Sum of linear and hyperbolic events on traces at ``offsets_m``."""
    out = np.zeros((n_traces, nt))
    for e in range(n_lin + n_hyp):
        amp = rng.normal()
        t0 = rng.uniform(0.2, 1.8)
        if e < n_lin:
            p = rng.uniform(-0.4, 0.4) * 1e-3  # s/m
            t = t0 + p * offsets_m
        else:
            v = rng.uniform(1500, 3500)
            t = np.sqrt(t0 ** 2 + (offsets_m / v) ** 2)
        ts = t * SAMPLES_PER_S
        if channel_shift is not None:
            ts = ts + channel_shift * rng.uniform(-2, 2)
        _add_events(out, ts, np.full(n_traces, amp))
    return out


def _add_noise(rng, x: np.ndarray, frac: float = 0.01) -> np.ndarray:
    rms = float(np.sqrt(np.mean(x * x))) if x.size else 0.0
    return x + frac * rms * rng.standard_normal(x.shape)


def blend_sum(shottimes, channels, trace_types, data, n_times):
    """Pseudo-deblended data: sum every non-missing trace into a continuous
    record per channel, zero the spans of bad traces, read each trace back at
    its own shot time (missing traces read back as zeros)."""
    all_st = np.concatenate(shottimes)
    all_ch = np.concatenate(channels)
    all_tt = np.concatenate(trace_types)
    t0 = int(all_st.min())
    t1 = int(all_st.max()) + max(n_times)
    chans = np.unique(all_ch[all_tt != MISSING]) if np.any(all_tt != MISSING) else np.array([], int)
    cidx = {int(c): i for i, c in enumerate(chans.tolist())}
    rec = np.zeros((max(len(chans), 1), t1 - t0))
    mute = np.zeros((max(len(chans), 1), t1 - t0), bool)
    for st, ch, tt, d, nt in zip(shottimes, channels, trace_types, data, n_times):
        d2 = d.reshape(-1, nt)
        for i in np.nonzero(tt != MISSING)[0]:
            c = cidx[int(ch[i])]
            s = int(st[i]) - t0
            rec[c, s: s + nt] += d2[i]
            if tt[i] == BAD:
                mute[c, s: s + nt] = True
    rec[mute] = 0.0
    out = []
    for st, ch, tt, d, nt in zip(shottimes, channels, trace_types, data, n_times):
        o = np.zeros((len(st), nt))
        for i in np.nonzero(tt != MISSING)[0]:
            c = cidx[int(ch[i])]
            s = int(st[i]) - t0
            o[i] = rec[c, s: s + nt]
        out.append(o.reshape(d.shape))
    return out


def gather_2d(seed: int = 1000, n_shots: int = 128, nt: int = 512,
              window=(32, 256), n_its: int = 100) -> Survey:
    """2-D common-receiver gather, one channel."""
    rng = np.random.default_rng(seed)
    offsets = (np.arange(n_shots) - n_shots // 2) * 12.5
    truth = _add_noise(rng, _events(rng, n_shots, offsets, nt))
    gaps = rng.uniform(0.8, 1.2, n_shots)
    st = np.round(np.cumsum(gaps) * SAMPLES_PER_S).astype(np.int64)
    ch = np.zeros(n_shots, np.int32)
    tt = np.zeros(n_shots, np.int32)
    truth = truth.astype(np.float32)
    data = blend_sum([st], [ch], [tt], [truth], [nt])[0].astype(np.float32)
    return Survey("gather_2d", [0], [2], [list(window)], [[0]], [[n_shots, nt]],
                  [st], [ch], [tt], [data], [truth], n_its)


def two_volume_3d(seed: int = 1001, n_ch: int = 64, n_shots: int = 128, nt: int = 1024,
                  window=(16, 32, 256), n_its: int = 200, bad_frac: float = 0.04,
                  missing_frac: float = 0.04) -> Survey:
    """Two disjoint source volumes of (channel, shot, time) with interleaved
    jittered shot times and two long gaps in the records."""
    rng = np.random.default_rng(seed)
    n_tr = n_ch * n_shots
    # shot times: volume A at 1.2 k + U[0, 0.5], volume B at 1.2 k + 0.6 + U[0, 0.5]
    ta = 1.2 * np.arange(n_shots) + rng.uniform(0, 0.5, n_shots)
    tb = 1.2 * np.arange(n_shots) + 0.6 + rng.uniform(0, 0.5, n_shots)
    merged = np.sort(np.concatenate([ta, tb]))
    conv_s = 5.12  # C * dt for the 1024-sample traces
    gap_after = [int(2 * n_shots * 85 / 256), int(2 * n_shots * 170 / 256)]
    bump = np.zeros_like(merged)
    for g in gap_after:
        bump[g + 1:] += 3.0 + conv_s
    lookup = dict(zip(merged.tolist(), (merged + bump).tolist()))
    ta = np.array([lookup[t] for t in ta.tolist()])
    tb = np.array([lookup[t] for t in tb.tolist()])
    shot_times = [np.round(ta * SAMPLES_PER_S).astype(np.int64),
                  np.round(tb * SAMPLES_PER_S).astype(np.int64)]
    ch_idx = np.repeat(np.arange(n_ch), n_shots)
    shot_idx = np.tile(np.arange(n_shots), n_ch)
    offsets = (shot_idx - n_shots // 2) * 12.5 + (ch_idx - n_ch // 2) * 25.0
    truths, sts, chs, tts = [], [], [], []
    for v in range(2):
        tr = _add_noise(rng, _events(rng, n_tr, offsets, nt, channel_shift=ch_idx))
        truths.append(tr.reshape(n_ch, n_shots, nt).astype(np.float32))
        sts.append(shot_times[v][shot_idx])
        chs.append(ch_idx.astype(np.int32))
        u = rng.uniform(size=n_tr)
        tt = np.full(n_tr, LIVE, np.int32)
        tt[u < bad_frac] = BAD
        tt[(u >= bad_frac) & (u < bad_frac + missing_frac)] = MISSING
        tts.append(tt)
    datas = blend_sum(sts, chs, tts, truths, [nt, nt])
    datas = [d.astype(np.float32) for d in datas]
    return Survey("two_volume_3d", [0, 1], [3, 3], [list(window), list(window)],
                  [[0, 0], [0, 0]], [[n_ch, n_shots, nt]] * 2, sts, chs, tts, datas,
                  truths, n_its)


def sweep(n: int = 256, f0: float = 8.0, f1: float = 80.0) -> np.ndarray:
    """Linear 8-80 Hz sweep over ``n`` samples with a cosine taper."""
    t = np.arange(n) * DT
    T = n * DT
    phase = 2 * np.pi * (f0 * t + 0.5 * (f1 - f0) / T * t * t)
    w = np.sin(phase)
    taper = np.ones(n)
    m = max(n // 10, 1)
    ramp = 0.5 * (1 - np.cos(np.pi * np.arange(m) / m))
    taper[:m] = ramp
    taper[n - m:] = ramp[::-1]
    return (w * taper).astype(np.float32)


def vibroseis_4d(seed: int = 1002, n_sy: int = 32, n_sx: int = 64, n_ch: int = 32,
                 nt: int = 2048, window=(16, 16, 16, 256), n_its: int = 150,
                 wavelet_len: int = 256) -> Survey:
    """(sourceY, sourceX, channel, time) volume whose traces are events
    convolved with one sweep; shot times in sY-major, sX-fast order."""
    rng = np.random.default_rng(seed)
    n_src = n_sy * n_sx
    n_tr = n_src * n_ch
    sy = np.repeat(np.arange(n_sy), n_sx * n_ch)
    sx = np.tile(np.repeat(np.arange(n_sx), n_ch), n_sy)
    ch = np.tile(np.arange(n_ch), n_src)
    off = np.sqrt(((sx - n_sx / 2) * 25.0) ** 2 + ((sy - n_sy / 2) * 25.0) ** 2) \
        + (ch - n_ch / 2) * 12.5
    spikes = _events(rng, n_tr, off, nt)
    wav = sweep(wavelet_len)
    nfft = nt + wavelet_len
    tr = np.fft.irfft(np.fft.rfft(spikes, nfft, axis=1) * np.fft.rfft(wav, nfft)[None],
                      nfft, axis=1)[:, :nt]
    tr = _add_noise(rng, tr).astype(np.float32)
    gaps = rng.uniform(0.8, 1.2, n_src)
    src_t = np.round(np.cumsum(gaps) * SAMPLES_PER_S).astype(np.int64)
    st = src_t[sy * n_sx + sx]
    tt = np.zeros(n_tr, np.int32)
    shape = [n_sy, n_sx, n_ch, nt]
    truth = tr.reshape(shape)
    data = blend_sum([st], [ch.astype(np.int32)], [tt], [truth], [nt])[0].astype(np.float32)
    return Survey("vibroseis_4d", [0], [4], [list(window)], [[0, 0, 0]], [shape], [st],
                  [ch.astype(np.int32)], [tt], [data], [truth], n_its,
                  wavelet_lengths=[wavelet_len], wavelet_idxs=[np.zeros(n_tr, np.int32)],
                  wavelets=[wav])


def uneven_gathers(n_gathers: int = 96, base_seed: int = 3000, n_its: int = 100):
    """Independent 2-D gathers with shots U{100..400}, time U{512..2048} and
    a window drawn from {(16,128), (32,256), (64,256)}."""
    out = []
    for g in range(n_gathers):
        rng = np.random.default_rng(base_seed + g)
        n_shots = int(rng.integers(100, 401))
        nt = int(rng.integers(512, 2049))
        window = [(16, 128), (32, 256), (64, 256)][int(rng.integers(0, 3))]
        out.append(gather_2d(seed=base_seed + g, n_shots=n_shots, nt=nt, window=window,
                             n_its=n_its))
    return out


def snr_db(out: list, truth: list, trace_types: list) -> float:
    """10 log10(sum true^2 / sum (out - true)^2) over live traces."""
    num = 0.0
    den = 0.0
    for o, t, tt in zip(out, truth, trace_types):
        nt = t.shape[-1]
        live = np.asarray(tt).reshape(-1) == LIVE
        o2 = np.asarray(o, np.float64).reshape(-1, nt)[live]
        t2 = np.asarray(t, np.float64).reshape(-1, nt)[live]
        num += float(np.sum(t2 * t2))
        den += float(np.sum((o2 - t2) ** 2))
    return 10.0 * np.log10(num / den) if den > 0 else float("inf")
