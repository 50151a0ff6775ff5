"""Benchmark of the deblending hot path: ISTA iterations per second.

Workloads (synthetic, seeded, agdeblend_b200.synthetic):
  two_volume_3d (default)  2 x (64 channels x 128 shots x 1024 samples)
      float32, windows (16, 32, 256), 8 % bad/missing traces, two 3 s record
      gaps, n_its 200;
  vibroseis_4d  32 sourceY x 64 sourceX x 32 channels x 2048 samples float32,
      one 256-sample 8-80 Hz sweep wavelet (trace length 2431), windows
      (16, 16, 16, 256), n_its 150;
  *_small  reduced versions of both (still larger than L2) for multi-pass
      ncu captures;
  uneven_gathers  96 independent 2-D receiver gathers (shots U{100..400},
      time U{512..2048}, windows from {(16,128), (32,256), (64,256)}), n_its
      100, solved together in one set of launches per iteration; compared
      with the same gathers solved one after another (per-gather loop).

One step = one ISTA iteration (forward operator, residual, adjoint, update,
soft threshold) over the whole survey.

  value  iterations/s with every input resident in HBM, CUDA events on the
         library's stream over exactly --steps iterations after --warmup;
  e2e    the same metric through the public agd_deblend call (host data in,
         planning, set-up, n_its iterations, output back to the host), the
         median of three timed calls after one untimed call;
  roofline  the dominant kernel of one profiled iteration against the
         measured HBM copy bandwidth;
  cpu_baseline  the reference's own OpenMP CPU path (oracle/_ref, built
         from the reference's sources) timed on this host.

Multi-GPU: the problem runs on one GPU, so N ranks run N independent replicas
(one survey each, different seeds); value = total iterations of all ranks /
max over ranks of the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

UNIT = "iterations/s"

# name -> (generator, keyword arguments, label of the metric)
WORKLOADS = {
    # the benchmark workload
    "two_volume_3d": ("two_volume_3d", dict(n_ch=64, n_shots=128, nt=1024),
                      "two-volume 3-D survey"),
    # the same survey at a quarter of the traces (model 167 MB, still larger
    # than L2): the case for multi-pass ncu captures
    "two_volume_3d_small": ("two_volume_3d", dict(n_ch=32, n_shots=64, nt=1024),
                            "two-volume 3-D survey, quarter size"),
    # the 4-D vibroseis survey with a source wavelet (model 10.4 GB)
    "vibroseis_4d": ("vibroseis_4d", dict(n_sy=32, n_sx=64, n_ch=32, nt=2048),
                     "4-D vibroseis survey with sweep wavelet"),
    # a quarter of its sources (9 windows, model 1.5 GB) for multi-pass ncu
    # captures
    "vibroseis_4d_small": ("vibroseis_4d", dict(n_sy=16, n_sx=32, n_ch=32, nt=2048),
                           "4-D vibroseis survey with sweep wavelet, quarter size"),
}
SEEDS = {"two_volume_3d": 1001, "vibroseis_4d": 1002}
# batches of independent problems: name -> (number of gathers, label)
BATCHES = {"uneven_gathers": (96, "96 uneven 2-D gathers solved together")}


def metric_label(name):
    return WORKLOADS[name][2] if name in WORKLOADS else BATCHES[name][1]


def metric_of(name):
    return f"ISTA iterations/s (plain FP32 deblending, {metric_label(name)})"


def workload(name="two_volume_3d", seed_offset=0):
    from agdeblend_b200 import synthetic as S

    gen, kw, _ = WORKLOADS[name]
    return getattr(S, gen)(seed=SEEDS[gen] + seed_offset, **kw)


def config_of(sv, name="two_volume_3d"):
    gen, w, _ = WORKLOADS[name]
    if gen == "two_volume_3d":
        desc = (f"{name}: 2 volumes x ({w['n_ch']} ch x {w['n_shots']} shots x "
                f"{w['nt']} samples) f32, windows (16,32,256), 4% bad + 4% missing "
                "traces, 2 record gaps")
    else:
        desc = (f"{name}: {w['n_sy']} sY x {w['n_sx']} sX x {w['n_ch']} ch x {w['nt']} "
                "samples f32, 256-sample 8-80 Hz sweep wavelet, windows (16,16,16,256)")
    return {"workload": desc, "n_its": sv.n_its, "initial_factor": sv.initial_factor,
            "l2": "inputs larger than L2"}


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = threading.Event()

    def start(self):
        """Starts nvidia-smi and waits (at most 3 s) for its first sample, so
        that a short timed region that follows is sampled too; the samples
        taken before the region (the device idle) are dropped."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self.first.wait(3.0)
            self.lines.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


PROFILES = {"two_volume_3d": "kernels_two_volume_3d_small.md",
            "vibroseis_4d": "kernels_vibroseis_4d_small.md"}


def profiled_traffic(kernel: str, name: str):
    """DRAM bytes per launch of `kernel` on workload `name`, scaled from the
    committed ncu summary of its small case (profiles/)."""
    import re

    if name not in PROFILES:
        return None
    path = os.path.join(ROOT, "profiles", PROFILES[name])
    try:
        text = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch\[" + re.escape(kernel) + r"\]\s*=\s*([0-9.eE+]+)",
                  text)
    return float(m.group(1)) if m else None


def physical_cores() -> int:
    """Physical cores of this host (logical CPUs when the split is unknown)."""
    try:
        import psutil

        n = psutil.cpu_count(logical=False)
        if n:
            return int(n)
    except Exception:
        pass
    return os.cpu_count() or 1


# The reference's OpenMP path runs with one thread per physical core; the
# variable must be set before the OpenMP runtime starts (the first load of the
# reference library).
os.environ.setdefault("OMP_NUM_THREADS", str(physical_cores()))

FFT_BACKEND = ("the project's FFTW3-API stand-in (oracle/fftw_shim): this image has no "
               "system FFTW3 library")


def cpu_reference_rate(sv, its: int, lib_name="libagdeblend_ref.so"):
    """Iterations/s of the reference's CPU path: time agd_deblend with
    n_its = 1 and 1 + its; the difference is `its` loop iterations."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from agdeblend_b200.capi import DeblendArgs

    import ref_bind

    if not ref_bind.available(lib_name):
        return None
    times = []
    for n in (1, 1 + its):
        args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                           sv.shottimes, sv.channels, sv.trace_types, sv.data,
                           sv.wavelet_lengths, sv.wavelet_idxs, sv.wavelets, dtype=np.float32)
        t0 = time.perf_counter()
        rc = ref_bind.ref_deblend(args, sv.initial_factor, n, 0, lib_name=lib_name)
        times.append(time.perf_counter() - t0)
        if rc:
            raise RuntimeError("reference agd_deblend failed")
    dt = max(times[1] - times[0], 1e-9)
    serial = lib_name.endswith("_serial.so")
    threads = 1 if serial else int(os.environ["OMP_NUM_THREADS"])
    return {"value": its / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"agd_deblend n_its=1 vs 1+{its} on the full workload (difference = "
                      f"{its} iterations, {dt:.1f} s), "
                      + ("serial build" if serial else
                         f"OpenMP over windows, OMP_NUM_THREADS={threads} (physical cores)"),
            "fft": FFT_BACKEND}


def cpu_port_rate(sv, its: int):
    """Fallback when the reference build is absent: the numpy oracle."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import agd_oracle as O

    plan = O.make_plan(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets)
    x = plan.zero_model()
    d = O.blend_input(plan, sv.data)
    t0 = time.perf_counter()
    for _ in range(its):
        r = O.forward(plan, x) - d
        g = O.adjoint(plan, r)
        x = O.threshold([xw - plan.step * gw for xw, gw in zip(x, g)], 0.0)
    dt = time.perf_counter() - t0
    return {"value": its / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{its} iterations of the float64 numpy oracle on the full workload"}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier_max(world, value):
    """Max of a per-rank value over all ranks (device tensor under NCCL,
    host tensor under gloo)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, args.steps)
    if args.workload in BATCHES:
        gathers = batch_workload(args.workload)
        config = batch_config(gathers, args.workload)
        res = cpu_batch_rate(gathers, 1)
        if res is None:
            res = {"value": float("nan"), "cores": 0, "kind": "port",
                   "sample": "reference build absent"}
    else:
        sv = workload(args.workload)
        config = config_of(sv, args.workload)
        res = cpu_reference_rate(sv, steps)
        if res is None:
            res = cpu_port_rate(sv, max(1, min(steps, 3)))
    line = {"impl": "reference", "metric": metric_of(args.workload), "value": res["value"],
            "unit": UNIT, "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": res["cores"],
                             "kind": res["kind"], "sample": res["sample"]},
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_single(args, name, rank, world, local, cpu_its):
    """One workload of one survey: the bench line of rank 0 (None elsewhere)."""
    import torch

    import agdeblend_b200 as A

    sv = workload(name, seed_offset=rank)
    torch.cuda.set_device(local)
    prob = A.Problem.from_survey(sv)
    tc_windows = prob.set_precision(args.precision) if args.precision else 0
    # warm-up + timed region (CUDA events inside the library, on its stream)
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t = prob.time_iterations(sv.data, sv.initial_factor, sv.n_its, args.warmup, args.steps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = barrier_max(world, float(t[0]))
    value = world * args.steps / (ms / 1e3)
    ms_fwd, ms_adj = float(t[1]), float(t[2])
    prof = prob.profile_iteration(1e-3)
    info = prob.info
    kn = prob.kernels()
    # the end-to-end calls below get the device arrays this handle held (the
    # library keeps them for the next problem on the device)
    prob.close()

    # e2e: the public agd_deblend call with host buffers, one full solve
    e2e_s, snr = float("nan"), None
    wavelet_kw = {}
    if sv.wavelets is not None:
        wavelet_kw = dict(wavelet_idxs=sv.wavelet_idxs, wavelets=sv.wavelets)
    def public_call(n_its, data):
        """The public API on host data: agd_deblend, or for a precision
        mode the extension calls (plan, set the mode, solve, release); the
        page-locked input is overwritten with the result."""
        if not args.precision:
            return A.deblend(sv.volumes, sv.window_shapes, sv.coords, sv.shottimes,
                             sv.channels, sv.trace_types, sv.initial_factor, n_its, 0, data,
                             overwrite_input=True, **wavelet_kw)
        p = A.Problem.from_survey(sv)
        p.set_precision(args.precision)
        res = p.solve(data, sv.initial_factor, n_its, overwrite_input=True)
        p.close()
        return res

    if not args.no_e2e:
        pinned = PinnedInput(sv.data)
        # one untimed call first: the first call in a process also pays the
        # one-time mapping of fresh device memory
        public_call(2, pinned.fresh())
        # three timed calls, the median counts (one call is a single sample of
        # host-side set-up time)
        calls = []
        for _ in range(3):
            bufs = pinned.fresh()  # the caller's input, outside the timed region
            torch.cuda.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            out = public_call(sv.n_its, bufs)
            torch.cuda.synchronize()
            calls.append(barrier_max(world, time.perf_counter() - t0))
        e2e_s = float(np.median(calls))
        from agdeblend_b200.synthetic import snr_db

        snr = snr_db(out, sv.truth, sv.trace_types)
    e2e_value = world * sv.n_its / e2e_s
    data_bytes = sum(d.nbytes for d in sv.data)

    M = int(info[1])
    Rn = int(info[2])
    peak, peak_kind = hbm_peak()
    # Algorithmic bytes per launch: the share of
    # B_iter = 3 M 8 + 4 R 4 each kernel is responsible for - the forward
    # space kernel reads the model once, the adjoint space kernel reads and
    # writes it once, the blend gather writes A x and reads d, the adjoint
    # time kernel reads the residual; the time-axis kernels move only
    # intermediates (0 algorithmic bytes).
    nf = int(prof[14])
    fast = int(info[8]) == 1
    wav = sv.wavelets is not None
    wav_fast = int(info[9]) == 1
    # phases named by the kernel family the set-up picked for them
    names = ((kn["space_fwd"], kn["time_fwd"], "blend_gather", kn["time_adj"], kn["space_adj"])
             if fast else
             ("axis_pass_fwd0", "time_c2r_ola", "blend_gather", "time_r2c", "axis_pass_adj_last"))
    if wav:
        # the adjoint time phase then also holds the wavelet correlation
        names = names[:3] + (names[3] + "+" + ("wavelet_fast" if wav_fast else "wavelet_apply"),
                             names[4])
    phases = {
        names[0]: (prof[6], 8.0 * M),
        names[1]: (prof[1], 0.0),
        names[2]: (prof[3], 4.0 * Rn * 2),
        names[3]: (prof[4], 4.0 * Rn),
        names[4]: (prof[10 + nf - 1], 16.0 * M),
    }
    if wav:
        phases["wavelet_fast" if wav_fast else "wavelet_apply"] = (prof[2], 0.0)
    dom = max(phases, key=lambda k: phases[k][0])
    dom_ms, dom_bytes = phases[dom]
    iter_bytes = 3 * 8.0 * M + 4 * 4.0 * Rn
    ms_iter = ms / args.steps
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_ms > 0 and dom_bytes > 0 else 0.0
    traffic = profiled_traffic(dom, name)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "algorithmic_bytes": dom_bytes, "peak_source": peak_kind,
                "phase_ms": {k: v[0] for k, v in phases.items()},
                "iteration_algorithmic_GB": iter_bytes / 1e9,
                "iteration_achieved_GBs": iter_bytes / (ms_iter / 1e3) / 1e9,
                "iteration_frac": iter_bytes / (ms_iter / 1e3) / 1e9 / peak}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_rate(sv, cpu_its) or cpu_port_rate(sv, 1)
        if cpu is not None and cpu["kind"] == "reference" and name == "two_volume_3d":
            serial = cpu_reference_rate(sv, 1, "libagdeblend_ref_serial.so")
            if serial is not None:
                cpu["serial"] = {k: serial[k] for k in ("value", "unit", "cores", "sample")}
    line = None
    if rank == 0:
        # kernels per iteration as the library counts them (space and time
        # kernels both ways per window class, generic passes, the blend
        # gather, the threshold-schedule step, wavelet kernels)
        launches = args.steps * int(info[14])
        line = {"metric": metric_of(name), "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_iter,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": config_of(sv, name),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "clocks": clk,
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": data_bytes / sv.n_its,
                        "d2h_bytes_per_step": data_bytes / sv.n_its,
                        "call_s": e2e_s, "n_its": sv.n_its, "snr_db": snr,
                        "input": "page-locked host arrays, overwritten with the result "
                                 "(overwrite_input=True), refilled outside the timed region"},
                "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "ms_forward_half": ms_fwd, "ms_adjoint_half": ms_adj}
        if args.precision:
            line["precision"] = {"mode": "split_bf16", "tc_windows": tc_windows}
            line["metric"] = line["metric"].replace("plain FP32", "split-BF16 space DFTs")
            line["dtype"] = "f32 + split-bf16 tensor cores"
    return line


def batch_workload(name, seed_offset=0):
    from agdeblend_b200 import synthetic as S

    n, _ = BATCHES[name]
    return S.uneven_gathers(n, base_seed=3000 + 1000 * seed_offset)


def batch_config(gathers, name):
    wins = sorted({tuple(g.window_shapes[0]) for g in gathers})
    return {"workload": f"{name}: {len(gathers)} 2-D gathers, shots U{{100..400}}, time "
                        f"U{{512..2048}}, windows {wins}, f32",
            "n_its": gathers[0].n_its, "initial_factor": 1.0, "gathers": len(gathers),
            "l2": "inputs larger than L2"}


def cpu_batch_rate(gathers, its: int):
    """Reference CPU path over the gathers: agd_deblend n_its = 1 and 1 + its
    per gather; one batch iteration = one iteration of every gather."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from agdeblend_b200.capi import DeblendArgs

    import ref_bind

    if not ref_bind.available("libagdeblend_ref.so"):
        return None
    total = 0.0
    for g in gathers:
        times = []
        for n in (1, 1 + its):
            args = DeblendArgs(g.volumes, g.n_dims, g.window_shapes, g.coords, g.shapes,
                               g.shottimes, g.channels, g.trace_types, g.data, dtype=np.float32)
            t0 = time.perf_counter()
            if ref_bind.ref_deblend(args, 1.0, n, 0):
                raise RuntimeError("reference agd_deblend failed")
            times.append(time.perf_counter() - t0)
        total += max(times[1] - times[0], 1e-9)
    threads = int(os.environ["OMP_NUM_THREADS"])
    return {"value": its / total, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"agd_deblend n_its=1 vs 1+{its} on each of the {len(gathers)} gathers "
                      f"(sum of differences {total:.1f} s), OpenMP over windows, "
                      f"OMP_NUM_THREADS={threads} (physical cores)",
            "fft": FFT_BACKEND}


def measure_batch(args, name, rank, world, local):
    """The batch workload: the bench line of rank 0 (None elsewhere)."""
    import torch

    import agdeblend_b200 as A

    gathers = batch_workload(name, seed_offset=rank)
    torch.cuda.set_device(local)
    n_its = gathers[0].n_its
    data = [d for g in gathers for d in g.data]
    prob = A.Problem.from_batch(gathers)
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t = prob.time_iterations(data, 1.0, n_its, args.warmup, args.steps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = barrier_max(world, float(t[0]))
    value = world * args.steps / (ms / 1e3)
    prof = prob.profile_iteration(1e-3)
    info = prob.info
    prob.close()  # its device arrays serve the calls below
    # the same gathers one after another (one problem handle each, the same
    # timed iterations): the per-gather launch loop
    loop_ms = 0.0
    for g in gathers:
        p1 = A.Problem.from_survey(g)
        loop_ms += float(p1.time_iterations(g.data, 1.0, n_its, args.warmup, args.steps)[0])
        p1.close()
    loop_ms = barrier_max(world, loop_ms)
    e2e_s = float("nan")
    if not args.no_e2e:
        kw = [dict(volumes=g.volumes, window_shapes=g.window_shapes, coords=g.coords,
                   shottimes=g.shottimes, channels=g.channels, trace_types=g.trace_types,
                   data=g.data) for g in gathers]
        A.deblend_batch(kw, 1.0, 2)
        calls = []
        for _ in range(3):  # median of three timed calls
            torch.cuda.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            A.deblend_batch(kw, 1.0, n_its)
            torch.cuda.synchronize()
            calls.append(barrier_max(world, time.perf_counter() - t0))
        e2e_s = float(np.median(calls))
    M, Rn = int(info[1]), int(info[2])
    peak, peak_kind = hbm_peak()
    phases = {"space_fwd": (prof[0], 8.0 * M), "time_fwd": (prof[1], 0.0),
              "blend_gather": (prof[3], 8.0 * Rn), "time_adj": (prof[4], 4.0 * Rn),
              "space_adj": (prof[5], 16.0 * M)}
    dom = max(phases, key=lambda k: phases[k][0])
    dom_ms, dom_bytes = phases[dom]
    iter_bytes = 3 * 8.0 * M + 4 * 4.0 * Rn
    ms_iter = ms / args.steps
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "algorithmic_bytes": dom_bytes,
                "peak_source": peak_kind, "phase_ms": {k: v[0] for k, v in phases.items()},
                "iteration_algorithmic_GB": iter_bytes / 1e9,
                "iteration_achieved_GBs": iter_bytes / (ms_iter / 1e3) / 1e9,
                "iteration_frac": iter_bytes / (ms_iter / 1e3) / 1e9 / peak}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_batch_rate(gathers, 1)
    line = None
    if rank == 0:
        data_bytes = sum(d.nbytes for d in data)
        line = {"metric": metric_of(name), "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_iter, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": batch_config(gathers, name),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "clocks": clk,
                "per_gather_loop": {"value": world * args.steps / (loop_ms / 1e3), "unit": UNIT,
                                    "ms_per_step": loop_ms / args.steps},
                "e2e": {"value": world * n_its / e2e_s, "unit": UNIT,
                        "h2d_bytes_per_step": data_bytes / n_its,
                        "d2h_bytes_per_step": data_bytes / n_its, "call_s": e2e_s,
                        "n_its": n_its},
                "gpu_launches": args.steps * int(info[14]), "roofline": roofline,
                "cpu_baseline": cpu, "window_classes_fast": int(info[15]),
                "windows_fast": int(info[16]), "windows": int(info[0])}
    return line


class PinnedInput:
    """Page-locked host copies of a survey's patches: the input buffers of
    the end-to-end calls, refilled from the survey before each call (outside
    the timed region) because the calls overwrite them with the result."""

    def __init__(self, data):
        import torch

        self.src = data
        self.bufs = [torch.empty(d.shape, dtype=torch.from_numpy(d[:0]).dtype,
                                 pin_memory=True).numpy() for d in data]

    def fresh(self):
        for b, d in zip(self.bufs, self.src):
            np.copyto(b, d)
        return self.bufs


# Time to SNR (the learned warm start): per benchmark survey, the network
# family it is trained on, the training size and epochs, the learning
# rate and whether it follows a cosine decay (chosen on the validation
# surveys: the decay helps the 2-D gathers; the vibroseis lines, 30 small
# surveys, do best with a constant 5e-4 - longer or faster training fits
# them closer and warm-starts the held-out survey worse), the survey, a
# held-out validation survey of the same family (other seed) and the
# warm-started schedules to try on it: (schedule length n, first
# iteration k), run as iterations [k, n) of the n-iteration schedule.  The
# threshold of iteration k depends on k / n, so a shorter schedule begun at
# the same fraction starts at the same level and descends faster.
def _schedules(lengths, counts):
    """(n, k) pairs running `c` iterations for c in counts, n in lengths."""
    return [(n, n - c) for c in counts for n in lengths if n - c >= 1]


TIME_TO_SNR = {
    "vibroseis_4d": ("vibroseis", 30, 12, 5e-4, False, lambda S: S.vibroseis_4d(seed=1002),
                     lambda S: S.vibroseis_4d(seed=4999),
                     _schedules((150, 100, 80, 60, 50, 40),
                                (10, 20, 25, 30, 35, 40, 45, 50, 55, 60, 75, 100))),
    "two_volume_3d": ("gather_2d", 2000, 8, 1e-3, True, lambda S: S.two_volume_3d(),
                      lambda S: S.two_volume_3d(seed=4998),
                      _schedules((200, 100, 60), (5, 10, 20, 25, 30, 40, 60, 80, 100))),
}


def timed(f):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = f()
    torch.cuda.synchronize()
    return r, time.perf_counter() - t0


def measure_time_to_snr(name):
    """Wall time of one public-API solve on host data (agd_gpu_solve for the
    plain method; agd_gpu_solve_learned - network estimate on the device,
    warm model, the tail of the same threshold schedule - for the learned
    start) until the deblended SNR against the known truth reaches the
    plain method's own final SNR minus 0.1 dB.  The learned start's
    schedule (its length and first iteration) is the candidate with the
    fewest iterations that reaches the plain method's SNR (-0.1 dB) on the
    validation survey; it is then used unchanged on the benchmark survey.
    Median of three calls each."""
    import agdeblend_b200 as A
    from agdeblend_b200 import synthetic as S
    from agdeblend_b200 import warmstart as WS

    family, n_train, epochs, lr, cosine, make, make_val, grid = TIME_TO_SNR[name]
    (net, losses), t_train = timed(lambda: WS.train(family, n_train, epochs=epochs, lr=lr,
                                                    cosine=cosine))

    def snr(out, sv):
        return S.snr_db(out, sv.truth, sv.trace_types)

    # the warm-started schedule, chosen on the validation survey: the first
    # of the candidates (fewest iterations first) reaching the plain
    # method's SNR there
    val = make_val(S)
    p = A.Problem.from_survey(val)
    target_val = snr(p.solve(val.data, val.initial_factor, val.n_its), val) - 0.1
    n_pick, k_pick = grid[-1]
    val_curve = {}
    for n, k in grid:
        val_curve[f"{n}:{k}"] = snr(
            WS.solve_learned(p, net, val.data, val.initial_factor, n, k), val)
        if val_curve[f"{n}:{k}"] >= target_val:
            n_pick, k_pick = n, k
            break
    p.close()

    sv = make(S)
    p = A.Problem.from_survey(sv)
    pinned = PinnedInput(sv.data)
    p.solve(pinned.fresh(), sv.initial_factor, 2, overwrite_input=True)  # device arrays, graphs
    WS.solve_learned(p, net, pinned.fresh(), sv.initial_factor, n_pick, n_pick,
                     overwrite_input=True)

    def median_call(f):
        """Three calls on a fresh page-locked copy of the input each (the
        copy outside the timed region); the call overwrites it."""
        runs = []
        for _ in range(3):
            bufs = pinned.fresh()
            runs.append(timed(lambda: f(bufs)))
        return [np.array(o) for o in runs[-1][0]], float(np.median([r[1] for r in runs]))

    plain, t_plain = median_call(
        lambda d: p.solve(d, sv.initial_factor, sv.n_its, overwrite_input=True))
    target = snr(plain, sv) - 0.1
    learned, t_learned = median_call(
        lambda d: WS.solve_learned(p, net, d, sv.initial_factor, n_pick, k_pick,
                                   overwrite_input=True))
    res = {"metric": "seconds to the plain method's deblended SNR - 0.1 dB (one solve, host "
                     "data in and out)", "unit": "s", "higher_is_better": False,
           "survey": name, "target_snr_db": target,
           "plain_fp32": {"seconds": t_plain, "iterations": sv.n_its - 1,
                          "snr_db": snr(plain, sv)},
           "learned_fp32": {"seconds": t_learned, "iterations": n_pick - k_pick,
                            "schedule": n_pick, "it_begin": k_pick, "snr_db": snr(learned, sv),
                            "reached": bool(snr(learned, sv) >= target)},
           "speedup_learned_fp32": t_plain / t_learned,
           "network": {"family": family, "training": n_train, "epochs": epochs,
                       "lr": lr, "cosine_lr": cosine, "input_channels": net.in_channels,
                       "loss_first_last": [float(losses[0]), float(losses[-1])],
                       "train_seconds": t_train},
           "validation": {"target_snr_db": target_val,
                          "snr_db_by_schedule_and_start": val_curve}}
    if name == "vibroseis_4d":
        # the precision variant: split-BF16 tensor-core space DFTs as well
        n_tc = p.set_precision(1)
        p.solve(pinned.fresh(), sv.initial_factor, 2, overwrite_input=True)
        lb, t_lb = median_call(
            lambda d: WS.solve_learned(p, net, d, sv.initial_factor, n_pick, k_pick,
                                       overwrite_input=True))
        pb, t_pb = median_call(
            lambda d: p.solve(d, sv.initial_factor, sv.n_its, overwrite_input=True))
        res["learned_split_bf16"] = {"seconds": t_lb, "iterations": n_pick - k_pick,
                                     "snr_db": snr(lb, sv), "reached": bool(snr(lb, sv) >= target),
                                     "tc_windows": n_tc}
        res["plain_split_bf16"] = {"seconds": t_pb, "snr_db": snr(pb, sv)}
        res["speedup_learned_split_bf16"] = t_plain / t_lb
    p.close()
    net.close()
    return res


SUMMARY_KEYS = ("metric", "value", "unit", "ms_per_step", "config", "clocks", "e2e",
                "gpu_launches", "roofline", "cpu_baseline", "per_gather_loop")


def workload_summary(line):
    return {k: line[k] for k in SUMMARY_KEYS if k in line}


# multiply-adds per level-0 pixel of the warm-start network with base c
# channels: 3 x 3 convolutions, level l on 4^-l of the pixels
def network_macs_per_pixel(c: int = 32) -> int:
    levels = [(1 * c + c * c + c * c + c * 1),
              (c * 2 * c + 4 * c * c + 4 * c * c + 2 * c * c),
              (2 * c * 4 * c + 16 * c * c + 16 * c * c + 4 * c * 2 * c),
              (4 * c * 8 * c + 8 * c * 4 * c)]
    return 9 * sum(m // 4 ** lv for lv, m in enumerate(levels))


def measure_network(steps: int = 5, warmup: int = 3, n: int = 64, h: int = 64, w: int = 2048):
    """Forward passes of the warm-start network (base 32) on seeded images
    through agd_nn_forward (host arrays in and out): pixels/s and the
    convolutions' TFLOP/s.  The default shape is one network pass of the
    vibroseis survey's estimate: 64 receiver lines of 64 shots x 2048
    samples (8.4 M pixels)."""
    import time

    import torch

    from agdeblend_b200.nn import WarmStartNet

    net = WarmStartNet(32, seed=0)
    x = np.random.default_rng(7).standard_normal((n, h, w)).astype(np.float32)
    for _ in range(warmup):
        net.forward(x)
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        net.forward(x)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    net.close()
    s = float(np.median(times))
    px = n * h * w
    return {"metric": "warm-start network forward, images in and out through host memory",
            "images": [n, h, w], "ms": 1e3 * s, "pixels_per_s": px / s,
            "conv_tflops": 2.0 * network_macs_per_pixel(32) * px / s / 1e12,
            "macs_per_pixel": network_macs_per_pixel(32)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-its", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1],
                    help="1: split-BF16 tensor-core space DFTs (agd_gpu_problem_set_precision)")
    ap.add_argument("--no-time-to-snr", action="store_true",
                    help="skip the learned warm-start time-to-SNR measurements")
    ap.add_argument("--time-to-snr-only", action="store_true",
                    help="only the time-to-SNR measurements (one JSON line)")
    ap.add_argument("--network-only", action="store_true",
                    help="only the warm-start network's forward throughput (one JSON line)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="only the headline workload (no vibroseis_4d / uneven_gathers entries)")
    ap.add_argument("--workload", default="two_volume_3d",
                    choices=sorted(WORKLOADS) + sorted(BATCHES))
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank, int(os.environ.get("WORLD_SIZE", "1")))
        return
    if args.network_only:
        print(json.dumps(measure_network()), flush=True)
        return
    if args.time_to_snr_only:
        print(json.dumps({n: measure_time_to_snr(n) for n in TIME_TO_SNR}), flush=True)
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.workload in BATCHES:
            line = measure_batch(args, args.workload, rank, world, local)
        else:
            line = measure_single(args, args.workload, rank, world, local, args.cpu_its)
        if (world == 1 and args.workload == "two_volume_3d" and not args.no_workloads
                and not args.precision and line is not None):
            # the other benchmark workloads, each measured the same way, in
            # the same JSON line
            line["workloads"] = {
                "vibroseis_4d": workload_summary(
                    measure_single(args, "vibroseis_4d", rank, world, local, 1)),
                "uneven_gathers": workload_summary(
                    measure_batch(args, "uneven_gathers", rank, world, local)),
            }
            if not args.no_time_to_snr:
                line["time_to_snr"] = {n: measure_time_to_snr(n) for n in TIME_TO_SNR}
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
