#!/usr/bin/env python
"""ViSQOL throughput on B200: pairs/s of the batched GPU pipeline.

A step scores one batch of audio-mode pairs (10 s, 48 kHz, the seeded
music-like generator of akvisqol_b200.synth, per-pair seeds) through the
C ABI. ``value`` times the batch with its signals already in HBM (device
inputs; CUDA events on the engine's stream, first launch to last result
copy); ``e2e`` times the public call with pinned host buffers, host-to-device
copies and result read-back included. Each step's inputs (~0.5 GB) exceed
the 126 MB L2, so no flush is needed between steps.

The headline form is --precision (fast: f32 gammatone stages; balanced:
f64 with FMA; exact: the CPU path's f64 operation order); the other forms
are timed the same way and reported under "forms", each with its largest
|dMOS| against the CPU model on the baseline sample.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--precision F]
  python bench.py --impl reference ...   # the reference CPU model (oracle), all host threads

With torchrun (N > 1) every rank scores its own batch (weak scaling, no
collective on the data path); the step time is the maximum over ranks. The
uneven batches and the serving sweep are one-GPU measurements and run at
N = 1 only.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRICS = {
    "fast": "ViSQOL pairs/s (audio mode, 10 s 48 kHz pairs), FP32 form, 1 B200",
    "balanced": "ViSQOL pairs/s (audio mode, 10 s 48 kHz pairs), FP64 FMA form, 1 B200",
    "exact": "ViSQOL pairs/s (audio mode, 10 s 48 kHz pairs), exact FP64 form, 1 B200",
}
DTYPES = {"fast": "f32 (gammatone stages 3-4 above the lowest band group, lag-search transform; rescoring, "
                  "NSIM, DP, MOS in f64)",
          "balanced": "f64 (FMA); the lag search's nominating transform in f32, its rescoring in f64",
          "exact": "f64; the lag search's nominating transform in f32, its rescoring in f64"}
# gammatone: pipe-peak kind of visqol_b200_peak and the algorithm's flops per
# sample, the same for every form: 4 biquads of 7 flops, the window multiply
# and the square-accumulate (reference src/gammatone.zig:268-306)
ROOF = {"exact": (0, 31.0, "fp64-pipe (mul/add)"), "balanced": (1, 31.0, "fp64-pipe (fma)"),
        "fast": (2, 31.0, "fp32-pipe (fma), stages 1-2 on the fp64 pipe")}
WORKLOAD = "audio-mode pairs, 10 s at 48 kHz (480,000 samples; degraded 481,776), seeded synthetic music-like generator"
# HBM copy bandwidth of this pool's B200s when the driver's measurement
# (MEASURED_PEAKS.json) is absent
HBM_FALLBACK_GBS = 6650.0


def hbm_peak() -> tuple[float, str]:
    """(GB/s, source) of the HBM roofline denominator."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.is_file():
        try:
            d = json.loads(f.read_text())
            for key in ("hbm_gbs", "hbm_GBps", "hbm"):
                if isinstance(d.get(key), (int, float)) and d[key] > 0:
                    return float(d[key]), f"of measured (MEASURED_PEAKS.json {key})"
        except (OSError, ValueError):
            pass
    return HBM_FALLBACK_GBS, "of fallback (6.65 TB/s, an earlier copy measurement on this pool)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--batch", type=int, default=128)
    p.add_argument("--seconds", type=float, default=10.0)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fast", choices=["fast", "balanced", "exact"])
    p.add_argument("--only", action="store_true", help="time the --precision form alone")
    p.add_argument("--serve-requests", type=int, default=5000,
                   help="requests per offered load in the serving sweep (0: skip the sweep)")
    p.add_argument("--config-pairs", type=int, default=256,
                   help="pairs per mode in the uneven-batch accuracy and throughput runs (0: skip)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def all_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def make_pairs(count: int, seconds: float, seed0: int):
    from akvisqol_b200 import synth
    return [synth.audio_pair(seed0 + i, seconds=seconds) for i in range(count)]


class Clocks:
    """nvidia-smi samples every 100 ms while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(pairs, seconds: float) -> dict:
    """The CPU model (oracle restatement of the reference CPU path) on a
    bounded sample, pair-parallel on every host thread."""
    import oracle
    threads = os.cpu_count() or 1
    sample = pairs[: max(1, min(len(pairs), threads))]
    t0 = time.perf_counter()
    res = oracle.measure_batch([p[0] for p in sample], [p[1] for p in sample], 48000, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": len(sample) / dt, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": f"{len(sample)} pairs of {seconds:g} s audio, one batch", "results": res}


def run_reference(args, rank, world):
    if rank != 0:
        return
    import oracle
    threads = os.cpu_count() or 1
    pairs = make_pairs(max(1, threads), args.seconds, 0x5EED_0000)
    refs, degs = [p[0] for p in pairs], [p[1] for p in pairs]
    for _ in range(args.warmup):
        oracle.measure_batch(refs, degs, 48000, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.measure_batch(refs, degs, 48000, threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.mean(times))
    value = len(pairs) / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRICS[args.precision], "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch_per_step": len(pairs), "note": "inputs exceed L2"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                         "sample": f"{len(pairs)} pairs of {args.seconds:g} s audio per step"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


SERVE_LOADS = (0.25, 0.5, 0.75, 1.0, 1.2)


def uneven_configs(native, torch, n: int, plain_exact: float) -> dict:
    """The uneven batches: n audio pairs (48 kHz, log-uniform 3-30 s, cutoff
    4-16 kHz, SNR 10-40 dB, delay 0-200 ms) and n speech pairs (16 kHz,
    2-15 s). Batched pairs/s per form (signals in HBM, one batch per mode),
    and per form the per-pair |dMOS| against the CPU model with agreement of
    global lags, patch indices (VAD in speech mode) and matched offsets."""
    import oracle
    from akvisqol_b200 import synth
    sets = {"audio": (native.MODE_AUDIO, 48000, synth.audio_batch(n, min_s=3.0, max_s=30.0)),
            "speech": (native.MODE_SPEECH, 16000, synth.speech_batch(n, min_s=2.0, max_s=15.0))}
    threads = os.cpu_count() or 1
    out = {}
    for name, (mode, sr, pairs) in sets.items():
        refs, degs = [p[0] for p in pairs], [p[1] for p in pairs]
        t0 = time.perf_counter()
        res = oracle.measure_batch(refs, degs, sr, oracle.options(mode=mode), threads=threads)
        cpu_s = time.perf_counter() - t0
        d_ref = [torch.from_numpy(r).cuda() for r in refs]
        d_deg = [torch.from_numpy(d).cuda() for d in degs]
        torch.cuda.synchronize()
        entry = {"pairs": n, "seconds_total": float(sum(r.size for r in refs)) / sr,
                 "cpu_model_pairs_per_s": n / cpu_s, "cpu_threads": threads}
        for form in ("exact", "balanced", "fast"):
            ctx = native.Context(mode=mode, use_lattice_model=False, precision=form)
            args = ([t.data_ptr() for t in d_ref], [t.data_ptr() for t in d_deg], sr)
            kw = dict(device_inputs=True, ref_lens=[t.numel() for t in d_ref], deg_lens=[t.numel() for t in d_deg])
            ctx.measure_batch_traced(*args, **kw)  # warm
            got = ctx.measure_batch_traced(*args, **kw)
            ms = ctx.last_timing()["total_ms"]
            dm = [abs(g[1]["moslqo"] - w[1]["moslqo"]) for g, w in zip(got, res) if g[0] == 0 and w[0] == 0]
            entry[form] = {"pairs_per_s": n / (ms / 1e3), "failures": sum(1 for g in got if g[0] != 0),
                           "max_abs_dmos": max(dm) if dm else None,
                           "p99_abs_dmos": float(np.percentile(dm, 99)) if dm else None,
                           "median_abs_dmos": float(np.median(dm)) if dm else None,
                           "pairs_over_1e-6": int(sum(1 for v in dm if v > 1e-6))}
            del ctx
        entry["exact_speedup_vs_plain_exact"] = entry["exact"]["pairs_per_s"] / plain_exact if mode == 0 else None
        # discrete decisions of every form against the CPU model on a subset (traces are per pair)
        k = min(n, 24)
        wtrs = [oracle.measure(r, d, sr, oracle.options(mode=mode))[1] for r, d in zip(refs[:k], degs[:k])]
        agree = {f: 0 for f in ("exact", "balanced", "fast")}
        for form in agree:
            ctx = native.Context(mode=mode, use_lattice_model=False, precision=form)
            got = ctx.measure_batch_traced(refs[:k], degs[:k], sr)
            for (c, _, tr), wtr in zip(got, wtrs):
                agree[form] += int(c == 0 and tr["global_lag"] == wtr["global_lag"]
                                   and list(tr["ref_index"]) == list(wtr["ref_index"])
                                   and list(tr["deg_offset"]) == list(wtr["deg_offset"])
                                   and list(tr["realign_lag"]) == list(wtr["realign_lag"]))
            del ctx
        entry["decisions_identical"] = {f: f"{v}/{k}" for f, v in agree.items()}
        out[name] = entry
        del d_ref, d_deg
    return out


def serve_sweep(native, torch, precision: str, pool, n_req: int, seed: int) -> dict:
    """Poisson arrivals of the serving mix (70% audio 48 kHz 2-60 s, 30%
    speech 16 kHz 2-20 s) into a visqol_b200_server, signals resident in
    HBM. Peak = pairs/s with every request queued at once; then each offered
    load (a fraction of that peak) runs n_req requests and reports achieved
    pairs/s and submit-to-result latency percentiles."""
    import threading
    rng = np.random.default_rng(seed)
    dev = [(mode, sr, torch.from_numpy(p[0]).cuda(), torch.from_numpy(p[1]).cuda()) for mode, sr, p in pool]
    audio = [i for i, d in enumerate(dev) if d[0] == 0]
    speech = [i for i, d in enumerate(dev) if d[0] == 1]
    torch.cuda.synchronize()

    server = native.Server(precision=precision, lanes=4, max_batch=64)

    def submit(i):
        mode, sr, r, d = dev[i]
        server.submit(mode, r.data_ptr(), d.data_ptr(), sr, device_inputs=True, ref_len=r.numel(), deg_len=d.numel())

    # warm-up: every pool pair once (engines, rate caches, FFT tables, arenas)
    for rep in range(2):
        for i in range(len(dev)):
            submit(i)
        for _ in range(len(dev)):
            server.next(timeout_ms=600000)
    server.stats(reset=True)

    def run(rate):
        picks = [audio[rng.integers(len(audio))] if rng.random() < 0.7 else speech[rng.integers(len(speech))]
                 for _ in range(n_req)]
        gaps = rng.exponential(1.0 / rate, n_req) if rate else np.zeros(n_req)
        failures = [0]

        def produce():
            t_next = time.perf_counter()
            for k, i in enumerate(picks):
                t_next += gaps[k]
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                submit(i)

        t0 = time.perf_counter()
        th = threading.Thread(target=produce)
        th.start()
        for _ in range(n_req):
            item = server.next(timeout_ms=600000)
            if item is None or item[1] != 0:
                failures[0] += 1
        wall = time.perf_counter() - t0
        th.join()
        st = server.stats(reset=True)
        return {"offered_pairs_per_s": rate, "pairs_per_s": n_req / wall, "latency_p50_ms": st["latency_p50_ms"],
                "latency_p99_ms": st["latency_p99_ms"], "queue_p99_ms": st["queue_p99_ms"],
                "mean_batch": st["mean_batch"], "failures": failures[0]}

    def saturate(window: int):
        """Closed loop: keep `window` requests outstanding; sustained pairs/s."""
        picks = [audio[rng.integers(len(audio))] if rng.random() < 0.7 else speech[rng.integers(len(speech))]
                 for _ in range(n_req)]
        t0 = time.perf_counter()
        sent = 0
        for _ in range(min(window, n_req)):
            submit(picks[sent])
            sent += 1
        for _ in range(n_req):
            server.next(timeout_ms=600000)
            if sent < n_req:
                submit(picks[sent])
                sent += 1
        wall = time.perf_counter() - t0
        server.stats(reset=True)
        return n_req / wall

    peak = saturate(4 * 64)
    loads = [dict(load=f, **run(f * peak)) for f in SERVE_LOADS]
    server.close()
    # capacity: the closed-loop probe, or the best rate an offered load sustained
    capacity = max([peak] + [l["pairs_per_s"] for l in loads if l["failures"] == 0])
    return {"requests_per_load": n_req, "peak_pairs_per_s": peak, "capacity_pairs_per_s": capacity,
            "peak_definition": "closed loop with lanes x max_batch = 256 requests outstanding", "loads": loads,
            "mix": "70% audio 48 kHz log-uniform 2-60 s, 30% speech 16 kHz log-uniform 2-20 s; "
                   f"{len(pool)} distinct seeded pairs resident in HBM, drawn per request",
            "lanes": 4, "max_batch": 64}


def serve_pool(seed0: int, n_audio: int = 70, n_speech: int = 30):
    from akvisqol_b200 import synth
    pool = [(0, 48000, p) for p in synth.audio_batch(n_audio, seed0=seed0, min_s=2.0, max_s=60.0)]
    pool += [(1, 16000, p) for p in synth.speech_batch(n_speech, seed0=seed0 + 0x8000, min_s=2.0, max_s=20.0)]
    return pool


def isolated_gammatone(native, form: str, ptr_r, ptr_d, len_r, len_d, warmup: int) -> dict:
    """The headline form's gammatone kernel with nothing else of the step
    beside it: one lane, references prepared beforehand, so the timed
    launches (degraded spectrograms, realigned frames) follow the lag phase
    on the lane's one stream. Same workload and batch as the timed steps."""
    prev = os.environ.get("VISQOL_GPU_LANES")
    os.environ["VISQOL_GPU_LANES"] = "1"
    try:
        ctx = native.Context(mode=native.MODE_AUDIO, precision=form)
    finally:
        if prev is None:
            os.environ.pop("VISQOL_GPU_LANES")
        else:
            os.environ["VISQOL_GPU_LANES"] = prev
    prep = ctx.prepare(ptr_r, 48000, device_inputs=True, ref_lens=len_r)

    def step():
        for o in ctx.measure_prepared(prep, ptr_d, device_inputs=True, deg_lens=len_d):
            if not isinstance(o, native.NativeError):
                native.free(o)
        return ctx.last_timing()

    for _ in range(max(1, warmup)):
        step()
    ts = [step() for _ in range(3)]
    kind, flops_per_sample, bound = ROOF[form]
    ms = sum(t["gammatone_kernel_ms"] for t in ts)
    rms = sum(t["gammatone_rms"] for t in ts)
    launches = sum(t["gammatone_launches"] for t in ts)
    achieved = flops_per_sample * ts[0]["gammatone_window"] * rms / (ms / 1e3) / 1e12 if ms > 0 else None
    peak = native.peak_tflops(kind)
    lag_ms = sum(t["lag_kernel_ms"] for t in ts)
    lag_bytes = sum(t["lag_bytes"] for t in ts)
    hbm, hbm_src = hbm_peak()
    lag_gbs = lag_bytes / (lag_ms / 1e3) / 1e9 if lag_ms > 0 else None
    del prep, ctx
    return {"achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved and peak else None,
            "launches": launches, "rms": rms, "kernel_ms": ms, "batches": len(ts),
            "lag_search": {"bound": "hbm", "achieved": lag_gbs, "peak": hbm, "unit": "GB/s",
                           "frac": lag_gbs / hbm if lag_gbs else None, "peak_source": hbm_src,
                           "bytes_per_batch": lag_bytes / len(ts), "kernel_ms_per_batch": lag_ms / len(ts),
                           "bytes": "signals read (twice in the f32 search: transform and rescoring) + four "
                                    "passes over the transform buffer (16 B a point in f64, 8 B in f32)"},
            "how": "one lane, prepared references: the degraded-signal and realignment launches, and the global lag "
                   "search, with no other kernel of the step beside them; CUDA events around each launch group"}


def run_ours(args, rank, world, local):
    os.environ["VISQOL_CUDA_DEVICE"] = str(local)
    import torch
    from akvisqol_b200 import native
    torch.cuda.set_device(local)
    B = args.batch
    pairs = make_pairs(B, args.seconds, 0x5EED_0000 + 1000003 * rank)
    forms = [args.precision] + ([] if args.only else [f for f in ("fast", "balanced", "exact") if f != args.precision])
    ctxs = {f: native.Context(mode=native.MODE_AUDIO, precision=f) for f in set(forms) | {"exact"}}
    # device-resident inputs (torch is only the allocator here)
    d_ref = [torch.from_numpy(r).cuda() for r, _ in pairs]
    d_deg = [torch.from_numpy(d).cuda() for _, d in pairs]
    ptr_r = [t.data_ptr() for t in d_ref]
    ptr_d = [t.data_ptr() for t in d_deg]
    len_r = [t.numel() for t in d_ref]
    len_d = [t.numel() for t in d_deg]
    torch.cuda.synchronize()

    def timed(form, clocks_box=None):
        ctx = ctxs[form]

        def dev_step():
            out = ctx.measure_batch_scores(ptr_r, ptr_d, 48000, device_inputs=True, ref_lens=len_r, deg_lens=len_d)
            return out, ctx.last_timing()

        for _ in range(args.warmup):
            dev_step()
        torch.cuda.synchronize()
        barrier(world)
        timings, walls, results = [], [], None
        with Clocks(local) as clocks:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                results, t = dev_step()
                walls.append(time.perf_counter() - t0)
                timings.append(t)
        torch.cuda.synchronize()
        barrier(world)
        dev_ms_max = all_max(sum(t["total_ms"] for t in timings), world)
        kind, flops_per_sample, bound = ROOF[form]
        gt_ms = sum(t["gammatone_kernel_ms"] for t in timings)
        gt_launches = sum(t["gammatone_launches"] for t in timings)
        gt_rms = sum(t["gammatone_rms"] for t in timings)
        window = timings[0]["gammatone_window"]
        achieved = flops_per_sample * window * gt_rms / (gt_ms / 1e3) / 1e12 if gt_ms > 0 else None
        peak = native.peak_tflops(kind)
        return {
            "value": world * B * args.steps / (dev_ms_max / 1e3), "ms_per_step": dev_ms_max / args.steps,
            "walls": walls, "timings": timings, "results": results, "clocks": clocks.summary(),
            "failures": sum(1 for c, _ in results if c != 0),
            "gt_rms": gt_rms, "gt_launches": gt_launches,
            "roofline": {"bound": bound, "kernel": "gammatone", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": (achieved / peak) if achieved and peak else None,
                         "flops_per_rms": flops_per_sample * window,
                         "peak_source": f"measured here: visqol_b200_peak kind {kind}"},
        }

    runs = {f: timed(f) for f in forms}
    head = runs[args.precision]
    ctx = ctxs[args.precision]

    # prepared references: the same batch scored against references prepared
    # once (outside the timed region), degraded signals in HBM
    prep = ctx.prepare(ptr_r, 48000, device_inputs=True, ref_lens=len_r)

    def prep_step():
        for o in ctx.measure_prepared(prep, ptr_d, device_inputs=True, deg_lens=len_d):
            if not isinstance(o, native.NativeError):
                native.free(o)
        return ctx.last_timing()

    for _ in range(args.warmup):
        prep_step()
    barrier(world)
    prep_ms = all_max(sum(prep_step()["total_ms"] for _ in range(args.steps)), world)
    prepared_line = {"value": world * B * args.steps / (prep_ms / 1e3), "unit": "pairs/s",
                     "ms_per_step": prep_ms / args.steps, "speedup_vs_direct": None}
    prepared_line["speedup_vs_direct"] = prepared_line["value"] / head["value"]
    del prep

    # e2e: public API, pinned host buffers, copies inside the timed region
    pin_r = [torch.from_numpy(r).pin_memory().numpy() for r, _ in pairs]
    pin_d = [torch.from_numpy(d).pin_memory().numpy() for _, d in pairs]
    for _ in range(args.warmup):
        for o in ctx.measure_batch(pin_r, pin_d, 48000):
            if not isinstance(o, native.NativeError):
                native.free(o)
    barrier(world)
    e2e_times, h2d, d2h = [], 0, 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        outs = ctx.measure_batch(pin_r, pin_d, 48000)
        moses = [o.contents.moslqo for o in outs if not isinstance(o, native.NativeError)]
        for o in outs:
            if not isinstance(o, native.NativeError):
                native.free(o)
        e2e_times.append(time.perf_counter() - t0)
        t = ctx.last_timing()
        h2d, d2h = t["h2d_bytes"], t["d2h_bytes"]
    e2e_s = all_max(float(np.sum(e2e_times)), world)
    e2e_value = world * B * args.steps / e2e_s

    # the same public call with every upload ahead of the scoring (no
    # overlap), for comparison
    os.environ["VISQOL_STREAMED_UPLOADS"] = "0"
    barrier(world)
    direct_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for o in ctx.measure_batch(pin_r, pin_d, 48000):
            if not isinstance(o, native.NativeError):
                native.free(o)
        direct_times.append(time.perf_counter() - t0)
    os.environ.pop("VISQOL_STREAMED_UPLOADS")
    direct_value = world * B * args.steps / all_max(float(np.sum(direct_times)), world)
    signal_bytes = sum(r.nbytes + d.nbytes for r, d in pairs)

    # The dominant kernel (gammatone) on its own: one lane, nothing of the
    # step beside it, so achieved = algorithmic flops / its own event-timed
    # duration. The in-step figure (launch spans that include other lanes'
    # kernels sharing the GPU) is kept under in_step.
    iso = isolated_gammatone(native, args.precision, ptr_r, ptr_d, len_r, len_d, args.warmup)
    in_step = dict(head["roofline"])
    in_step["how"] = ("in the timed steps: every lane's launches share the GPU with the other lanes' kernels, so "
                      "each launch's event-timed span (and this fraction) includes that sharing")
    roof = {"bound": in_step["bound"], "kernel": "gammatone", "achieved": iso["achieved"], "peak": iso["peak"],
            "unit": "TFLOP/s", "frac": iso["frac"], "flops_per_rms": in_step["flops_per_rms"],
            "peak_source": in_step["peak_source"], "traffic": None,
            "kernel_ms_per_batch": iso["kernel_ms"] / iso["batches"], "rms_per_batch": iso["rms"] / iso["batches"],
            "how": iso["how"], "lag_search": iso["lag_search"], "in_step": in_step}
    prof = ROOT / "profiles" / "gammatone_traffic.json"
    if prof.is_file():
        per_rms = json.loads(prof.read_text()).get("dram_bytes_per_rms_audio48k")
        if per_rms:
            roof["traffic"] = per_rms * iso["rms"] / max(1, iso["launches"])
    timings = head["timings"]
    stage = {k: float(np.mean([t[k] for t in timings])) for k in
             ("lag_ms", "spectrogram_ms", "prep_ms", "nsim_ms", "realign_ms", "gammatone_kernel_ms", "total_ms")}

    # plain exact form: one pair per call
    plain = []
    for i in range(min(4, B)):
        t0 = time.perf_counter()
        o = ctxs["exact"].measure(pin_r[i], pin_d[i], 48000)
        native.free(o)
        plain.append(time.perf_counter() - t0)
    plain_value = 1.0 / float(np.mean(plain))

    walls = head["walls"]
    line = {
        "metric": METRICS[args.precision], "value": head["value"], "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPES[args.precision], "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch_per_gpu": B, "global_batch": world * B,
                   "inputs": "device-resident for value; pinned host for e2e",
                   "l2": "inputs (~0.5 GB per step) exceed L2; no flush", "precision": args.precision},
        "latency_ms": {"batch_p50": 1e3 * float(np.percentile(walls, 50)),
                       "batch_p99": 1e3 * float(np.percentile(walls, 99)),
                       "plain_single_pair_p50": 1e3 * float(np.percentile(plain, 50))},
        "plain_exact_pairs_per_s": plain_value,
        "speedup_vs_plain_exact": head["value"] / plain_value,
        "stage_ms": stage,
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "signal_bytes_per_step": int(signal_bytes),
                "uploads": "chunked, each chunk's upload overlapping the previous chunk's scoring",
                "value_uploads_first": direct_value},
        "gpu_launches": int(sum(t["kernel_launches"] for t in timings)),
        "clocks": head["clocks"],
        "failures": head["failures"],
        "forms": {f: {"value": r["value"], "ms_per_step": r["ms_per_step"], "roofline": r["roofline"],
                      "failures": r["failures"]} for f, r in runs.items()},
        "prepared_references": prepared_line,
        "autotune": native.autotune_choices(),
    }
    # The uneven batches and the serving sweep are one-GPU measurements: a
    # multi-rank run (weak scaling of the batch step) leaves them to N = 1.
    if args.config_pairs > 0 and rank == 0 and world == 1:
        line["uneven_batches"] = uneven_configs(native, torch, args.config_pairs, plain_value)
    if args.serve_requests > 0 and world == 1:
        pool = serve_pool(0x5EED_4000 + 7919 * rank)
        line["serving"] = {f: serve_sweep(native, torch, f, pool, args.serve_requests, 17 + rank)
                           for f in dict.fromkeys([args.precision, "balanced", "exact"])}
        del pool
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(pairs, args.seconds)
        res = cb.pop("results")
        line["cpu_baseline"] = cb
        # parity on every pair of the timed batch: the rest of it through the
        # CPU model too (untimed)
        if len(res) < len(pairs):
            import oracle
            rest = pairs[len(res):]
            res = res + oracle.measure_batch([p[0] for p in rest], [p[1] for p in rest], 48000,
                                             threads=os.cpu_count() or 1)
        for f, r in runs.items():
            dmos = [abs(o["moslqo"] - g[1]) for (c, o), g in zip(res, r["results"]) if c == 0 and g[0] == 0]
            line["forms"][f]["max_abs_dmos_vs_oracle"] = max(dmos) if dmos else None
            line["forms"][f]["parity_pairs"] = len(dmos)
        line["parity"] = {"pairs": line["forms"][args.precision]["parity_pairs"],
                          "max_abs_dmos_vs_oracle": line["forms"][args.precision]["max_abs_dmos_vs_oracle"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        # Rank 0 alone times the CPU model; other ranks exit without work.
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, world, local = dist_setup()
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
