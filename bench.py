#!/usr/bin/env python3
"""Throughput of the spektri filter bank + Welch spectrum on B200.

Metric: input Msamples/s.  Workload (default): the batching configuration —
a real int16 stream at 64.8 MS/s, forward FFT 65536 with 25 % overlap, Welch
average over 256 blocks, 256 channels with IFFT sizes 64..8192 and taper
widths 8..64, 64 blocks per buffer.  A step is one buffer (64 blocks,
3,145,728 new samples) through the whole path: forward FFTs, Welch terms and
accumulation, and the filter bank (one persistent launch).

  value : device-resident input and outputs, CUDA events on the launching
          stream over K steps (max over ranks), inputs cycled over more than
          L2 of distinct buffers and outputs (200 MB/step) larger than L2.
  e2e   : the public host API (sk_process): pinned host input copied in, all
          channel outputs and spectra copied back, every step; its bound is
          the pinned device-to-host copy bandwidth, measured and reported.
  plain_value: the plain per-channel path (one filter-bank launch per
          channel) on the same buffers; batched_over_plain is the ratio.
  roofline: the filter-bank kernel, algorithmic bytes (its channel outputs)
          per launch / its span inside the batched graph (device timestamps),
          against the measured HBM copy bandwidth.
  roofline_pipeline: the whole step's algorithmic bytes (input + channel
          outputs) / the step time, against the same bandwidth.
  cpu_baseline: the FP32 CPU restatement of the reference path on this host's
          cores, on a bounded sample of the same workload.

``--impl reference`` times that CPU restatement alone (the reference arm:
the Rust reference cannot be built without a Rust toolchain).
Multi-GPU (torchrun): each rank processes its own stream of the same
configuration (replicas, weak scaling); no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DISTINCT_BUFFERS = 48          # 48 x 6.3 MB of input cycled: 302 MB > 126 MB L2


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "window": "from the untimed pre-roll through the end of the timed region"}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, ws, local):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(w, raws, seconds, threads):
    """The FP32 CPU restatement on a bounded sample: whole buffers of the same
    workload until ``seconds`` of work (at least 2 buffers)."""
    from oracle import oracle32
    o = oracle32.Oracle32(w.fs, w.fc, w.fft_size, w.ffts_per_buf, w.averages, w.fmt, w.filters(),
                          spectrum_format="f32", n_threads=threads)
    o.process(raws[0])                        # warm-up (thread start, page faults)
    n = 0
    t0 = time.perf_counter()
    while True:
        o.process(raws[n % len(raws)])
        n += 1
        dt = time.perf_counter() - t0
        if (dt >= seconds and n >= 2) or n >= 400:
            break
    return n * w.samples_per_buffer / dt, n


def workload_config(w, ws):
    """The workload as both arms report it (identical dicts: the same
    configuration is measured on the GPU and on the host cores)."""
    return {"workload": w.name, "input": w.fmt, "fs": w.fs, "fft_size": w.fft_size,
            "ffts_per_buf": w.ffts_per_buf, "averages": w.averages, "channels": len(w.channels),
            "sum_ifft_bins": sum(c["n"] for c in w.channels), "samples_per_step": w.samples_per_buffer,
            "parallelism": f"replicas x{ws}"}


def d2h_copy_gbs(dev, nbytes=256 << 20, reps=5):
    """Pinned device-to-host copy bandwidth (GB/s), best of ``reps`` copies
    timed with CUDA events: the bound of the host path's output copies."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    dst = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    best = 0.0
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize(dev)
        best = max(best, nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


def run_reference(args, ws, rank):
    """Reference arm: the CPU restatement with all host threads, on this
    workload's configuration; each step one bounded sample (a buffer)."""
    if rank != 0:
        return
    from spektri_b200 import workloads
    from oracle import oracle32
    w = workloads.WORKLOADS[args.workload]()
    if args.ffts_per_buf:
        w.ffts_per_buf = args.ffts_per_buf
    threads = len(os.sched_getaffinity(0))
    per_buf = w.samples_per_buffer
    raw = workloads.stream_numpy(w, 0, 2 * per_buf)
    raws = [r.view(np.uint8) for r in np.split(raw, 2)]
    o = oracle32.Oracle32(w.fs, w.fc, w.fft_size, w.ffts_per_buf, w.averages, w.fmt, w.filters(),
                          spectrum_format="f32", n_threads=threads)
    for i in range(args.warmup):
        o.process(raws[i % 2])
    t0 = time.perf_counter()
    for i in range(args.steps):
        o.process(raws[i % 2])
    dt = time.perf_counter() - t0
    v = args.steps * per_buf / dt / 1e6
    line = {
        "impl": "reference", "metric": "input Msamples/s", "value": round(v, 3), "unit": "Msamples/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(w, ws),
        "cpu_baseline": {"value": round(v, 3), "unit": "Msamples/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} buffers of {per_buf} samples (FP32 C++ restatement; the Rust "
                                   f"reference needs a Rust toolchain, absent here)"},
        "e2e": {"value": round(v, 3), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--mode", default="batched", choices=["batched", "plain"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip timing the plain per-channel path (one filter-bank launch per channel)")
    ap.add_argument("--ffts-per-buf", type=int, default=0, help="override blocks per buffer (small profiling cases)")
    ap.add_argument("--preroll", type=float, default=1.5, help="seconds of untimed steps while clocks are sampled")
    ap.add_argument("--tuning", default="", help="SIZE,THREADS,CTAS_PER_SM: fixed filter-bank tile shape instead of autotuning")
    ap.add_argument("--adjoint", action="store_true",
                    help="also time the differentiable forward and the adjoint (always on for c4)")
    ap.add_argument("--by-size", action="store_true",
                    help="also time the filter bank of each IFFT size alone (same tile shape)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return

    import torch
    from spektri_b200 import Plan, pinned_empty, workloads

    dev = local
    torch.cuda.set_device(dev)
    w = workloads.WORKLOADS[args.workload]()
    if args.ffts_per_buf:
        w.ffts_per_buf = args.ffts_per_buf
    w.seed += 7919 * rank                                 # each replica its own stream
    spb = w.samples_per_buffer
    nbuf = min(DISTINCT_BUFFERS, w.n_samples // spb)
    stream_dev = workloads.stream_torch(w, nbuf * spb, f"cuda:{dev}")
    raw_bytes = spb * w.bytes_per_sample
    raws = [stream_dev[i * raw_bytes:(i + 1) * raw_bytes] for i in range(nbuf)]

    def make(mode):
        return Plan(w.fs, w.fft_size, w.fmt, w.filters(), fc_in=w.fc, ffts_per_buf=w.ffts_per_buf,
                    averages=w.averages, spectrum_format="f32", mode=mode, device=dev)

    plan = make(args.mode)
    if args.tuning:
        plan.set_tuning(*[int(v) for v in args.tuning.split(",")])
        tile_size, tile_threads, ctas_per_sm, tune_us = plan.tuning() + (None,)
    else:
        tile_size, tile_threads, ctas_per_sm, tune_us = plan.autotune()   # cached per device / FFT size / channel mix
    outs = [torch.empty(c["out_samples"], dtype=torch.complex64, device=dev) for c in plan.channels]
    spec = torch.empty(plan.max_spectra * plan.spectrum_bytes, dtype=torch.uint8, device=dev)
    st = torch.cuda.Stream(dev)

    def run_steps(p, k, start):
        with torch.cuda.stream(st):
            for i in range(k):
                p.process_device(raws[(start + i) % nbuf], outs, spec, stream=st)

    run_steps(plan, args.warmup, 0)
    torch.cuda.synchronize(dev)
    # Clock samples: the sampler starts during an untimed pre-roll of the same
    # steps (>= 1 s, so nvidia-smi has samples under load) and runs to the end
    # of the timed region.
    clocks = ClockSampler(dev)
    clocks.start()
    t_pre = time.perf_counter()
    k_pre = 0
    while time.perf_counter() - t_pre < args.preroll:
        run_steps(plan, 20, k_pre)
        torch.cuda.synchronize(dev)
        k_pre += 20
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    run_steps(plan, args.steps, args.warmup)
    e1.record(st)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, ws, local)
    value = args.steps * spb * ws / (ms_max / 1e3) / 1e6       # Msamples/s, all ranks

    # Stage spans in the production path (the same graph and buffers): device
    # timestamps of each kernel's first start / last end per call.  The
    # filter bank's span (Welch end -> filter-bank end, the dependent-launch
    # gap included) is the roofline's launch time.
    kt = min(args.steps, 50)
    plan.set_trace(True)
    run_steps(plan, kt, 0)
    trace_ms, tcalls = plan.trace()
    plan.set_trace(False)
    # The same stages launched one by one under CUDA events (no graph, no
    # dependent launches): a cross-check of the spans.
    plan.set_timing(True)
    run_steps(plan, kt, 0)
    stage_ms, calls = plan.timing()
    plan.set_timing(False)
    fcfb_ms = trace_ms[2] / max(1, tcalls)
    out_bytes = sum(c["out_samples"] for c in plan.channels) * 8
    hbm, peak_kind = peaks()
    achieved = out_bytes / (fcfb_ms / 1e3) / 1e9
    alg = w.alg_bytes_per_sample()
    # FP32 work of the same launch: per block and channel an n-point complex
    # FFT (5 n log2 n) plus the weight product (6 n); chirp-z sizes count two
    # M-point FFTs and three pointwise products.
    flops = 0.0
    for c in plan.channels:
        n = c["bins"]
        if n & (n - 1) == 0:
            flops += 5.0 * n * math.log2(n) + 6.0 * n
        else:
            m = 1 << math.ceil(math.log2(n + 6 * (n // 8) - 1))
            flops += 2 * 5.0 * m * math.log2(m) + 18.0 * m
    flops *= w.ffts_per_buf
    props = torch.cuda.get_device_properties(dev)
    fp32_peak = props.multi_processor_count * 128 * 2 * (clk.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
    result = {
        "metric": "input Msamples/s", "value": round(value, 2), "unit": "Msamples/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded int16 noise + tones + noise carriers, generated on the GPU)",
        "config": workload_config(w, ws),
        "mode": args.mode,
        "tuning": {"tile_size": tile_size, "tile_threads": tile_threads, "ctas_per_sm": ctas_per_sm,
                   "fcfb_us": round(tune_us, 1) if tune_us else None, "source": "fixed" if args.tuning else "autotuned"},
        "l2": f"{nbuf} distinct input buffers cycled ({nbuf * raw_bytes / 1e6:.0f} MB) and "
              f"{out_bytes / 1e6:.0f} MB of outputs per step, both above the 126 MB L2",
        "alg_bytes_per_sample": round(alg, 3),
        # the whole step (forward FFT, Welch, filter bank under the graph):
        # input bytes + channel-output bytes per sample x samples/s
        "roofline_pipeline": {"bound": "hbm", "achieved": round(value * 1e6 / ws * alg / 1e9, 1), "peak": hbm,
                              "unit": "GB/s", "frac": round(value * 1e6 / ws * alg / 1e9 / hbm, 4),
                              "peak_kind": f"{peak_kind} copy bandwidth",
                              "alg_bytes_per_step": round(alg * spb)},
        "stage_ms": {k: round(v / max(1, tcalls), 4) for k, v in zip(["fwd_fft", "welch", "fcfb"], trace_ms)},
        "stage_ms_source": "device timestamps inside the batched graph (sk_plan_trace), mean over "
                           f"{tcalls} calls",
        "stage_ms_direct": {k: round(v / max(1, calls), 4) for k, v in zip(["fwd_fft", "welch", "fcfb"], stage_ms)},
        "roofline": {"bound": "hbm", "kernel": "fcfb_kernel (persistent)", "achieved": round(achieved, 1),
                     "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "peak_kind": f"{peak_kind} copy bandwidth", "traffic": None,
                     "alg_bytes_per_launch": out_bytes, "launch_ms": round(fcfb_ms, 4),
                     "launch_ms_source": "filter-bank span in the batched graph (device timestamps)",
                     "fp32": {"flop_per_launch": round(flops), "achieved_tflops": round(flops / (fcfb_ms / 1e3) / 1e12, 2),
                              "peak_tflops": round(fp32_peak, 1), "frac": round(flops / (fcfb_ms / 1e3) / 1e12 / fp32_peak, 4),
                              "peak_kind": "SMs x 128 FP32 lanes x 2 x max SM clock"}},
        "gpu_launches": plan.launches_per_call * args.steps,
        "clocks": clk,
    }
    prof = os.path.join(ROOT, "profiles", "fcfb_traffic.json")
    if os.path.exists(prof):
        d = json.load(open(prof))
        if d.get("workload") == w.name and d.get("kernel") == "fcfb_kernel":
            result["roofline"]["traffic"] = d.get("dram_bytes_per_launch")

    if not args.no_plain and args.mode == "batched":
        # The plain per-channel path (the reference's loop over filters,
        # fcfb.rs:66-100: one filter-bank launch per channel), same tile
        # shape, same buffers, same events: the batched path's speed-up.
        pp = make("plain")
        pp.set_tuning(tile_size, tile_threads, ctas_per_sm)
        run_steps(pp, args.warmup, 0)
        torch.cuda.synchronize(dev)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        kp = min(args.steps, 50)
        run_steps(pp, kp, 0)
        a1.record(st)
        torch.cuda.synchronize(dev)
        vp = kp * spb / (a0.elapsed_time(a1) / 1e3) / 1e6
        result["plain_value"] = round(vp * ws, 2)
        result["plain_launches_per_step"] = pp.launches_per_call
        result["batched_over_plain"] = round(value / ws / vp, 2)
        del pp

    if args.workload == "c4" or args.adjoint:
        # The differentiable stage on the same buffers: the filter bank as a
        # separate forward (sk_fcfb_forward_device) and its adjoint
        # (sk_fcfb_backward_device: dW and dX), input samples per second.
        K = plan.result_bins
        X = torch.empty(w.ffts_per_buf, K, dtype=torch.complex64, device=dev)
        win = torch.empty(plan.total * w.bytes_per_sample, dtype=torch.uint8, device=dev)
        win[:raw_bytes] = raws[0]
        win[raw_bytes:] = raws[1][: win.numel() - raw_bytes]
        plan.spectra_window_device(win, X, stream=st)
        W = [torch.from_numpy(plan.get_weights(i)).to(dev) for i in range(plan.n_channels)]
        ys = [torch.empty(c["out_samples"], dtype=torch.complex64, device=dev) for c in plan.channels]
        dys = [torch.randn(c["out_samples"], dtype=torch.complex64, device=dev) for c in plan.channels]
        dW = [torch.empty_like(x) for x in W]
        dX = torch.zeros_like(X)
        ka = min(args.steps, 50)

        def timed(fn):
            for _ in range(3):
                fn()
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record(st)
            for _ in range(ka):
                fn()
            b1.record(st)
            torch.cuda.synchronize(dev)
            return b0.elapsed_time(b1) / ka

        ms_f = timed(lambda: plan.fcfb_forward_device(X, W, ys, stream=st))
        ms_b = timed(lambda: plan.fcfb_backward_device(X, W, dys, dW, dX, stream=st))
        result["differentiable"] = {"fwd_value": round(spb / (ms_f / 1e3) / 1e6, 2),
                                    "bwd_value": round(spb / (ms_b / 1e3) / 1e6, 2), "unit": "Msamples/s",
                                    "fwd_ms": round(ms_f, 4), "bwd_ms": round(ms_b, 4),
                                    "what": "filter bank on one buffer's spectra: forward, and adjoint (dW + dX)"}

    if args.by_size:
        # Each IFFT size alone: a plan holding only that size's channels, the
        # same tile shape, its filter-bank launch timed under CUDA events.
        # Each figure includes one launch's fixed cost (claims, tail).
        by = {}
        for n in sorted({c["n"] for c in w.channels}):
            fl = [f for f, c in zip(w.filters(), w.channels) if c["n"] == n]
            ps = Plan(w.fs, w.fft_size, w.fmt, fl, fc_in=w.fc, ffts_per_buf=w.ffts_per_buf,
                      averages=w.averages, spectrum_format="f32", mode="batched", device=dev)
            try:
                ps.set_tuning(tile_size, tile_threads, ctas_per_sm)
            except Exception:
                ps.autotune()
            o2 = [torch.empty(c["out_samples"], dtype=torch.complex64, device=dev) for c in ps.channels]
            with torch.cuda.stream(st):
                for i in range(args.warmup):
                    ps.process_device(raws[i % nbuf], o2, spec, stream=st)
                ps.set_timing(True)
                for i in range(min(args.steps, 50)):
                    ps.process_device(raws[i % nbuf], o2, spec, stream=st)
            torch.cuda.synchronize(dev)
            sm_, nc = ps.timing()
            by[str(n)] = {"channels": len(fl), "points": len(fl) * n * w.ffts_per_buf,
                          "fcfb_us": round(sm_[2] / max(1, nc) * 1e3, 2)}
            del ps, o2
        result["fcfb_by_size"] = by

    # End to end through the public host API, with pinned host buffers.
    ke = max(1, min(args.e2e_steps, args.steps))
    nin = 4
    hin = [pinned_empty((raw_bytes,), np.uint8) for _ in range(nin)]
    for i in range(nin):
        hin[i][:] = raws[i].cpu().numpy()
    houts, hspec = plan.empty_outputs(pinned=True)
    plan.process_into(hin[0], houts, hspec)               # warm-up
    d2h = 0
    barrier(ws)
    t0 = time.perf_counter()
    for i in range(ke):
        r = plan.process_into(hin[i % nin], houts, hspec)
        d2h += out_bytes + r.n_spectra * plan.spectrum_bytes
    dt = time.perf_counter() - t0
    dt = max_over_ranks(dt, ws, local)
    d2h_peak = d2h_copy_gbs(dev)
    d2h_gbs = d2h / dt / 1e9
    result["e2e"] = {"value": round(ke * spb * ws / dt / 1e6, 2), "unit": "Msamples/s",
                     "h2d_bytes_per_step": raw_bytes, "d2h_bytes_per_step": int(d2h / ke),
                     # the host path copies every channel output back (alg bytes per sample x samples):
                     # its bound is the pinned device-to-host copy bandwidth, measured here
                     "d2h_gbs": round(d2h_gbs, 2), "d2h_peak_gbs": round(d2h_peak, 2),
                     "d2h_frac": round(d2h_gbs / d2h_peak, 4),
                     "api": "sk_process (pinned host input and outputs, one synchronous call per buffer)"}

    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0))
        raws_h = [hin[i].copy() for i in range(2)]
        v, n = cpu_baseline(w, raws_h, args.cpu_seconds, threads)
        result["cpu_baseline"] = {"value": round(v / 1e6, 3), "unit": "Msamples/s", "cores": threads,
                                  "kind": "port",
                                  "sample": f"{n} buffers x {spb} samples of the same workload, FP32 C++ "
                                            f"restatement, {threads} threads"}
    if rank == 0:
        print(json.dumps(result), flush=True)
    barrier(ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
