#!/usr/bin/env python3
"""Benchmark of the B200 Recon path (one JSON line on stdout, rank 0).

Workload (the batched configuration): 32 frames of uneven size per step --
16 x 1920x1080 and 16 x 3840x2160 YUV420P10, same-size 4:2:0 -> 4:4:4,
alternating algo 2 and algo 6, lanczos taps=4, sparse=1, qgate=1.0 -- on
seeded synthetic polygon frames (seed = base + frame index, offset per rank).

  value        whole-job output-luma Mpix/s of the batched form (one launch per
               stage over all 32 frames, CUDA graph replay), inputs resident in
               HBM, CUDA events on the launching stream, max over ranks
  e2e          same metric through the per-frame C ABI (lgcr_recon_frame) with
               pinned host planes: H2D, run, D2H inside the timed region, one
               calling host thread per core (at most 16) like fmParallel,
               the K steps' frames taken from one continuous queue
               (e2e_pageable: the same with pageable host planes); its
               copy_roofline is the step's H2D/D2H bytes over this box's
               measured duplex pinned-copy rate
  per_frame    device-resident per-frame path (one lgcr_recon_frame per frame)
  roofline     dominant stage: algorithmic bytes of the frames its launch
               processes (9 B per output pixel for 10-bit 4:2:0 -> 4:4:4) / its
               CUDA-event duration (separate event-bracketed pass) vs measured
               HBM; for the guided stage also counted FP32 FLOPs vs nominal FP32
  legs         the 1080p algo 2 batch (batched vs per-frame target) and the
               plain 720p, jinc resize and bm+bp configurations: batched and
               per-frame Mpix/s, stage split, roofline
  filters      Sharpen and TRecon (trad 1) per-frame device path on a 1080p
               clip and Downsample (quality 0/1/2) on 1080p 4:4:4 frames,
               beside the reference's AVX2 build on one thread
  cpu_baseline the reference's AVX2 build on this host's cores (bounded sample)
  serving      the serving configuration's mixed stream (5 frame kinds, algo
               2/4/6, bm on 10 %, 24 streams) into the continuous-batching
               server (8 GB budget): an arrival-rate sweep over server shapes
               names the highest rate with p99 <= 100 ms, then the full stream
               arrives (Poisson) at 1.2x the per-frame path's capacity on that
               shape: throughput and p50/p99/p99.9 latency

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import collections
import ctypes
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "vapoursynth-lgcr_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

from lgcr import replicas as R  # noqa: E402
from lgcr import synthetic as S  # noqa: E402  (numpy only; no GPU)

METRIC = "Recon 4:4:4 Mpix/s batched vs per-frame on 1 B200 at ≤1 LSB; p50/p99 ms"
WORKLOAD = ("batched 32 frames: 16x1920x1080 + 16x3840x2160 YUV420P10 -> 4:4:4 same size, "
            "algo 2/6 alternating, lanczos taps=4, sparse=1, qgate=1.0")
FILTER_ARGS = dict(kernel="lanczos", taps=4, sparse=1, qgate=1.0)
BYTES_PER_PIXEL = 9.0          # (1 + 2 * 1/4) * 2 B in + 3 * 2 B out per output pixel


def frame_specs(rank: int, frames: int = 32):
    """The workload's frames; `frames` < 32 keeps an equal number of 1080p and
    4K frames from the front of each half (smaller cases for profilers)."""
    specs = []
    half = max(1, frames // 2)
    for i in range(32):
        if i % 16 >= half:
            continue
        w, h = (1920, 1080) if i < 16 else (3840, 2160)
        specs.append(dict(index=i, width=w, height=h, algo=2 if i % 2 == 0 else 6,
                          seed=R.frame_seed(1000, rank, i)))
    return specs


def _gen(spec):
    return S.make_frame(spec["width"], spec["height"], S.YUV420P10, seed=spec["seed"])


def generate(specs, workers=None):
    # spawn pool before any CUDA call in this process
    workers = workers or min(len(specs), max(1, (os.cpu_count() or 2) - 1), 16)
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        return pool.map(_gen, specs)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix=f"lgcr_clocks_rank{index}_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            with open(self.path) as fh:
                rows = [r.split(",") for r in fh.read().strip().splitlines() if r.strip()]
            os.unlink(self.path)
        except Exception:
            return None
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# reference arm: the reference's AVX2 CPU build on the host cores
# ---------------------------------------------------------------------------
def host_cpu():
    """CPU model and logical core count of this host (for the CPU baselines)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "host_logical_cores": os.cpu_count() or 1,
            "usable_cores": cpu_threads()}


def cpu_threads():
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        n = os.cpu_count() or 1
    return max(1, min(n, 32))


def interleaved(specs):
    """Workload order alternating 1080p and 4K frames, so any prefix samples
    both sizes and both algorithms in proportion."""
    small = [s["index"] for s in specs if s["width"] == 1920]
    large = [s["index"] for s in specs if s["width"] != 1920]
    order = []
    for a, b in zip(small, large):
        order += [a, b]
    return order


def frame_queue(n, rounds, nthreads, work, latencies):
    """Call work(i) for every i in range(n), `rounds` times over, from
    `nthreads` threads taking the items from one continuous queue -- the way
    a VapourSynth host keeps requesting frames: a thread that finishes one
    step's last frame takes the next step's first instead of waiting for the
    slowest thread at a step boundary. Each call's latency (ms) is appended
    to `latencies`."""
    lock = threading.Lock()
    queue = collections.deque(i for _ in range(rounds) for i in range(n))

    def worker():
        while True:
            with lock:
                if not queue:
                    return
                i = queue.popleft()
            t0 = time.perf_counter()
            work(i)
            with lock:
                latencies.append(1000 * (time.perf_counter() - t0))

    ts = [threading.Thread(target=worker) for _ in range(nthreads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()


def run_cpu(frames, specs, steps, warmup, threads, per_step, min_seconds=0.0):
    """Each step: `per_step` frames (round-robin over the interleaved
    workload) across `threads` workers, one frame per worker at a time
    (fmParallel-like). Steps repeat until `min_seconds` of timed work."""
    from oracle import oracle as O
    filters = {}
    for spec in specs:
        key = (spec["width"], spec["height"], spec["algo"])
        if key not in filters:
            fmt = O.make_format(frames[spec["index"]], 10)
            filters[key] = [O.Recon(fmt, "avx2", algo=spec["algo"], **FILTER_ARGS)
                            for _ in range(threads)]
    times, pixels = [], []
    cursor = 0
    sequence = interleaved(specs)
    step = 0
    while step < warmup + steps or sum(times) < min_seconds:
        order = [sequence[(cursor + k) % len(sequence)] for k in range(per_step)]
        cursor += per_step
        lock = threading.Lock()
        queue = list(order)

        def worker(tid):
            while True:
                with lock:
                    if not queue:
                        return
                    i = queue.pop(0)
                spec = specs[i]
                f = filters[(spec["width"], spec["height"], spec["algo"])][tid]
                f.frame(frames[i], -1)

        t0 = time.perf_counter()
        ts = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        dt = time.perf_counter() - t0
        if step >= warmup:
            times.append(dt)
            pixels.append(sum(specs[i]["width"] * specs[i]["height"] for i in order))
        step += 1
    total_s = sum(times)
    return sum(pixels) / total_s / 1e6, total_s, times


def reference_scene_420ps(width=1920, height=1080):
    """The reference benchmark's own source (test/benchmark.py:131-168): a
    vertical edge, a diagonal and a low-amplitude texture in float 4:4:4,
    here box-averaged 2x2 to 4:2:0 (the reference converts with
    resize.Bilinear; the scene's structure, and so its sparse-active share,
    is the same)."""
    import numpy as np
    yy, xx = np.mgrid[0:height, 0:width]
    edge = (xx > width // 2).astype(np.float32)
    diagonal = (xx * height > yy * width).astype(np.float32)
    texture = (0.01 * np.sin(xx * 0.071) * np.cos(yy * 0.053)).astype(np.float32)
    y = (0.2 + 0.25 * edge + 0.03 * diagonal + texture).astype(np.float32)
    u = (-0.25 + 0.55 * edge + 0.5 * texture).astype(np.float32)
    v = (0.30 - 0.60 * edge - 0.5 * texture).astype(np.float32)
    box = lambda p: (0.25 * (p[0::2, 0::2] + p[1::2, 0::2] + p[0::2, 1::2] + p[1::2, 1::2])).astype(np.float32)
    return y, box(u), box(v)


def reference_scene_fps(seconds=3.0):
    """Single-thread time per frame of the reference's AVX2 build on its own
    benchmark scene at 1080p, algo 2, lanczos3, sparse, beside the published
    figures (Ryzen 9 5950X): ties this harness to the reference's numbers."""
    from oracle import oracle as O
    if not O.available("avx2"):
        return None
    planes = reference_scene_420ps()
    f = O.Recon(O.make_format(planes), "avx2", algo=2, kernel="lanczos", taps=3, sparse=1)
    f.frame(planes)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        f.frame(planes)
        n += 1
    fps = n / (time.perf_counter() - t0)
    _, st = f.frame(planes)
    return {"ms_per_frame_1_thread": round(1000.0 / fps, 2),
            "published_ms_per_frame_1_thread": 89.8,
            "published_source": "test/baselines/lgcr-cpu-optimized-1080p.jsonl (latency mode); "
                                "25.2 fps in the 1-thread throughput run, RELEASE_NOTES.md:19-28",
            "sparse_active_ratio": round(st.sparse_active_ratio, 4), "published_sparse_active": 0.058,
            "published_cpu": "AMD Ryzen 9 5950X", "scene": "1920x1080 YUV420PS edge/diagonal/texture",
            "args": "algo 2, lanczos taps=3, sparse=1", "build": "reference AVX2 (oracle/_ref)"}


# published 1-thread latency-mode ms per frame of the reference (Ryzen 9
# 5950X, test/baselines/lgcr-cpu-optimized-{1080p,4k}.jsonl)
PUBLISHED_SCENE_MS = {(1920, 1080): {2: 89.8, 4: 102.3, 6: 117.4},
                      (3840, 2160): {2: 229.5, 4: 271.7, 6: 367.4}}


def reference_scene_leg(dev, stream, frames=10):
    """The reference's own benchmark scene at 1080p and 4K, algo 2/4/6,
    lanczos3, sparse: device-path and host-path (per-frame C ABI, host
    planes, one caller) milliseconds per frame beside the reference's
    published single-thread figures."""
    import numpy as np
    import torch
    out = {}
    for (w, h), published in PUBLISHED_SCENE_MS.items():
        planes = reference_scene_420ps(w, h)
        dplanes = [torch.from_numpy(p).to(dev) for p in planes]
        for algo, ref_ms in published.items():
            f = lgcr.Recon(lgcr.format_of(planes), algo=algo, kernel="lanczos", taps=3, sparse=1)
            douts = [None] + [torch.empty((h, w), dtype=torch.float32, device=dev) for _ in range(2)]
            for _ in range(3):
                f.frame(dplanes, -1, out=douts, stream=stream.cuda_stream)
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(frames):
                f.frame(dplanes, -1, out=douts, stream=stream.cuda_stream)
            b.record(stream)
            torch.cuda.synchronize(dev)
            dev_ms = a.elapsed_time(b) / frames
            hout = [None] + [np.empty((h, w), np.float32) for _ in range(2)]
            f.frame(planes, -1, out=hout)
            lat = []
            for _ in range(frames):
                t0 = time.perf_counter()
                f.frame(planes, -1, out=hout)
                lat.append(1000 * (time.perf_counter() - t0))
            out[f"{w}x{h} algo{algo}"] = {"device_ms": round(dev_ms, 3),
                                          "host_call_ms": round(statistics.median(lat), 3),
                                          "reference_published_ms": ref_ms}
            f.close()
    return {"scene": "the reference's benchmark scene (edge/diagonal/texture), YUV420PS, "
                     "lanczos taps=3, sparse=1", "frames": out}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    specs = frame_specs(0)
    from oracle import oracle as O
    if not O.available("avx2"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/liblgcr_ref_avx2.so (the reference's AVX2 build) is missing"}))
        return 0
    threads = cpu_threads()
    frames = generate(specs)
    per_step = threads
    value, total_s, times = run_cpu(frames, specs, args.steps, args.warmup, threads, per_step)
    sample = (f"{per_step} frames per step ({threads} threads, one frame per thread, frames taken "
              f"round-robin from the 32-frame workload), reference AVX2 build (oracle/_ref)")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mpix/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * total_s / max(1, args.steps), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": WORKLOAD, "frames_per_step": per_step},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mpix/s", "cores": threads,
                         "kind": "reference", "sample": sample, **host_cpu()},
        "e2e": {"value": round(value, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# serving leg: the mixed request stream of the serving configuration
# ---------------------------------------------------------------------------
SERVE_KINDS = [
    ("1280x720 YUV420P8", 1280, 720, S.YUV420P8, {}, {}),
    ("1920x1080 YUV422P10", 1920, 1080, S.YUV422P10, {}, {}),
    ("3840x2160 YUV420P10", 3840, 2160, S.YUV420P10, {}, {}),
    ("1920x1080 YUV444PS", 1920, 1080, S.YUV444PS, {"blur_chroma": True}, {}),
    ("1920x1080->3840x2160 YUV420P10 jinc", 1920, 1080, S.YUV420P10, {},
     {"kernel": "jinc", "taps": 3, "width": 3840, "height": 2160}),
]
SERVE_STREAMS = 24
SERVE_SEEDS = 4          # content seeds per frame kind shared by the streams
SERVE_RING = 16          # host output buffers per kind


def _gen_serve(task):
    k, seed = task
    _, w, h, fmt, gen, _ = SERVE_KINDS[k]
    return S.make_frame(w, h, fmt, seed=seed, **gen)


def serve_requests(n, seed=4000):
    """(stream, kind, algo, bm) per request; bm on 10 % of them."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(SERVE_STREAMS)), int(rng.integers(len(SERVE_KINDS))),
             int(rng.choice([2, 4, 6])), bool(rng.random() < 0.1)) for _ in range(n)]


def serving_leg(frames, n_requests, lanes=2, max_batch=8, budget=8 << 30,
                sweep_factors=(0.5, 0.7, 0.9, 1.1), sweep_requests=600,
                sweep_servers=((2, 8), (2, 4), (3, 2))):
    """Shorter streams at several arrival rates and server shapes, then the
    full stream as Poisson arrivals at 1.2x the per-frame path's capacity on
    the shape that sustained the highest rate; latency from submit to
    completion on the server's clock."""
    import numpy as np
    import torch
    import lgcr

    def pinned_like(a):
        t = torch.empty(a.shape, dtype={np.uint8: torch.uint8, np.uint16: torch.int16,
                                        np.float32: torch.float32}[a.dtype.type], pin_memory=True)
        v = t.numpy()
        return v.view(a.dtype) if a.dtype == np.uint16 else v

    pins = {}
    for (k, s), planes in frames.items():
        pp = [pinned_like(p) for p in planes]
        for d, src in zip(pp, planes):
            d[...] = src
        pins[(k, s)] = pp
    filters, rings, ring_next = {}, {}, {}
    reqs = serve_requests(n_requests)

    def filt(k, algo, bm):
        key = (k, algo, bm)
        if key not in filters:
            _, w, h, fmt, _, fa = SERVE_KINDS[k]
            filters[key] = lgcr.Recon(lgcr.format_of(frames[(k, 0)], None if fmt.is_float else fmt.bits),
                                      algo=algo, bm=int(bm), **fa)
        return filters[key]

    def out_set(k):
        if k not in rings:
            f = filt(k, 2, False)
            same = f.out_w == SERVE_KINDS[k][1] and f.out_h == SERVE_KINDS[k][2]
            rings[k] = [[None if (p == 0 and same) else pinned_like(np.empty((f.out_h, f.out_w), f.dtype))
                         for p in range(3)] for _ in range(SERVE_RING)]
            ring_next[k] = 0
        i = ring_next[k]
        ring_next[k] = (i + 1) % SERVE_RING
        return i, rings[k][i]

    # warm-up: tables and workspaces of every filter the stream uses
    for (_, k, algo, bm) in {(0, k, a, b) for (_, k, a, b) in reqs}:
        filt(k, algo, bm).frame(pins[(k, 0)], -1, out=out_set(k)[1])
    # capacity of the per-frame path (one calling thread) on the stream's mix
    sample = reqs[:min(100, len(reqs))]
    t0 = time.perf_counter()
    for (s, k, algo, bm) in sample:
        filt(k, algo, bm).frame(pins[(k, s % SERVE_SEEDS)], -1, out=out_set(k)[1])
    plain_fps = len(sample) / (time.perf_counter() - t0)

    def run_stream(stream_reqs, rate, seed, n_lanes=lanes, batch_cap=max_batch):
        """Poisson arrivals at `rate` frames/s; per-request latency from submit
        to completion on the server's clock."""
        arrivals = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, len(stream_reqs)))
        server = lgcr.Server(budget_bytes=budget, max_batch=batch_cap, lanes=n_lanes,
                             queue_capacity=len(stream_reqs) + 1)
        tickets = [None] * len(stream_reqs)
        owner = {}                     # (kind, ring slot) -> request index using it
        infos = [None] * len(stream_reqs)
        pixels = 0
        start = time.perf_counter()
        for i, (st, k, algo, bm) in enumerate(stream_reqs):
            delay = start + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            slot, out = out_set(k)
            prev = owner.get((k, slot))
            if prev is not None and infos[prev] is None:
                infos[prev] = server.wait(tickets[prev])[1]      # ring slot still in flight
            owner[(k, slot)] = i
            f = filt(k, algo, bm)
            tickets[i] = server.submit(f, pins[(k, st % SERVE_SEEDS)], out)
            if tickets[i] < 0:
                raise RuntimeError(f"serving submit failed: {tickets[i]}")
            pixels += f.out_w * f.out_h
        for i in range(len(stream_reqs)):
            if infos[i] is None:
                infos[i] = server.wait(tickets[i])[1]
        server.close()
        lat = np.array([inf.done_ms - inf.submit_ms for inf in infos])
        span_ms = max(inf.done_ms for inf in infos) - min(inf.submit_ms for inf in infos)
        return {
            "arrival_rate_fps": round(rate, 1), "requests": len(stream_reqs),
            "failed": sum(1 for inf in infos if inf.status != 0),
            "throughput_fps": round(len(stream_reqs) / (span_ms / 1000), 1),
            "throughput_mpix_s": round(pixels / (span_ms / 1000) / 1e6, 1),
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                           "p99": round(float(np.percentile(lat, 99)), 3),
                           "p99.9": round(float(np.percentile(lat, 99.9)), 3)}}

    # arrival-rate sweep over server shapes: the highest rate whose p99 stays
    # under 100 ms is the sustainable throughput of this mixed stream
    sweep = []
    for (n_lanes, batch_cap) in sweep_servers:
        for factor in sweep_factors:
            r = run_stream(reqs[:sweep_requests], factor * plain_fps, 4100 + int(100 * factor),
                           n_lanes, batch_cap)
            r.update(rate_factor=factor, lanes=n_lanes, max_batch=batch_cap)
            sweep.append(r)
    ok = [r for r in sweep if r["latency_ms"]["p99"] <= 100.0 and r["failed"] == 0]
    best = max(ok, key=lambda r: r["throughput_mpix_s"]) if ok else None
    # the full stream at 1.2x capacity, on the server shape the sweep sustained best
    lanes, max_batch = (best["lanes"], best["max_batch"]) if best else (lanes, max_batch)
    main = run_stream(reqs, 1.2 * plain_fps, 4001, lanes, max_batch)
    return dict(main, **{
        "streams": SERVE_STREAMS,
        "kinds": [kd[0] for kd in SERVE_KINDS], "algos": [2, 4, 6], "bm_fraction": 0.1,
        "content": f"{SERVE_SEEDS} seeded frames per kind shared by the streams",
        "per_frame_capacity_fps": round(plain_fps, 1),
        "server": {"lanes": lanes, "max_batch": max_batch, "budget_gb": budget / 2 ** 30},
        "sweep": sweep,
        "sustainable_p99_under_100ms": ({"arrival_rate_fps": best["arrival_rate_fps"],
                                         "throughput_mpix_s": best["throughput_mpix_s"],
                                         "lanes": best["lanes"], "max_batch": best["max_batch"],
                                         "latency_ms": best["latency_ms"]} if best else None)})


# ---------------------------------------------------------------------------
# the other two filters of the plugin: Sharpen and TRecon on 1080p frames
# ---------------------------------------------------------------------------
FILTERS_CLIP = 6                 # frames of the 1080p YUV420P10 clip (TRecon trad 1)


def _gen_clip(task):
    import numpy as np
    seed, frames = task
    base = S.make_frame(1920 + 32, 1080 + 32, S.FrameFormat(10, 0, 0), seed=seed)
    rng = np.random.default_rng(seed)
    out = []
    for k in range(frames):
        mx, my = int(rng.integers(-3, 4)), int(rng.integers(-3, 4))
        planes = [p[16 + my:16 + my + 1080, 16 + mx:16 + mx + 1920].astype(np.float64)
                  for p in base]
        planes[1] = 0.25 * (planes[1][0::2, 0::2] + planes[1][1::2, 0::2] +
                            planes[1][0::2, 1::2] + planes[1][1::2, 1::2])
        planes[2] = 0.25 * (planes[2][0::2, 0::2] + planes[2][1::2, 0::2] +
                            planes[2][0::2, 1::2] + planes[2][1::2, 1::2])
        out.append(tuple(np.clip(np.rint(p), 0, 1023).astype(np.uint16) for p in planes))
    return out


def filters_leg(clip, dev, stream, steps, warmup):
    """Per-frame device-path throughput of Sharpen and TRecon (trad 1, every
    frame with its two neighbours) on a 1080p YUV420P10 clip resident in HBM,
    and of Downsample (quality 0, 1, 2) on 1080p YUV444P10 frames, beside the
    reference's AVX2 build on one host thread for one frame."""
    import numpy as np
    import torch
    from oracle import oracle as O
    fmt = lgcr.video_format(1920, 1080, 10, 1, 1)
    dclip = [[torch.from_numpy(p.view(np.int16)).to(dev).view(torch.uint16) for p in f]
             for f in clip]
    outs = [torch.empty((1080, 1920), dtype=torch.int16, device=dev).view(torch.uint16)
            for _ in range(3)]
    souts = [torch.empty_like(p) for p in dclip[0]]
    sharpen = lgcr.Sharpen(fmt)
    trecon = lgcr.TRecon(fmt, len(clip))
    h = stream.cuda_stream

    def sharpen_pass():
        for f in dclip:
            sharpen.frame(f, out=souts, stream=h)

    def trecon_pass():
        for n in range(len(dclip)):
            trecon.frame(n, lambda i: dclip[i], out=outs, stream=h)

    def timed(fn, frames):
        for _ in range(max(warmup, 1)):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms = a.elapsed_time(b) / (steps * frames)
        return {"ms_per_frame": round(ms, 3), "mpix_s": round(1920 * 1080 / (ms / 1000) / 1e6, 1)}

    res = {}
    for name, fn in (("sharpen", sharpen_pass), ("trecon", trecon_pass)):
        res[name] = {"workload": f"1920x1080 YUV420P10, {len(dclip)}-frame clip" +
                                 (", trad 1 (two neighbours)" if name == "trecon" else ""),
                     **timed(fn, len(dclip))}
    # Downsample: 4:4:4 -> 4:2:0 of 1080p 10-bit frames (Mpix/s of source pixels)
    f444 = S.FrameFormat(10, 0, 0)
    ds_clip = [S.make_frame(1920, 1080, f444, seed=7000 + i) for i in range(4)]
    ds_dev = [[torch.from_numpy(p.view(np.int16)).to(dev).view(torch.uint16) for p in f]
              for f in ds_clip]
    ds_out = [None] + [torch.empty((540, 960), dtype=torch.int16, device=dev).view(torch.uint16)
                       for _ in range(2)]
    for q in (0, 1, 2):
        ds = lgcr.Downsample(lgcr.video_format(1920, 1080, 10, 0, 0), quality=q)
        res[f"downsample_q{q}"] = {
            "workload": f"1920x1080 YUV444P10 -> 4:2:0, quality {q}, spline36, strength 1, "
                        f"{len(ds_dev)}-frame clip",
            **timed(lambda: [ds.frame(f, out=ds_out, stream=h) for f in ds_dev], len(ds_dev))}
        ds.close()
    if O.available("avx2"):
        t0 = time.perf_counter()
        O.sharpen(clip[1], 10, variant="avx2")
        res["sharpen"]["cpu_reference_ms_per_frame"] = round(1000 * (time.perf_counter() - t0), 1)
        t0 = time.perf_counter()
        O.trecon(clip[1], [clip[0], clip[2]], 10, len(clip), variant="avx2")
        res["trecon"]["cpu_reference_ms_per_frame"] = round(1000 * (time.perf_counter() - t0), 1)
        for q in (0, 1, 2):
            t0 = time.perf_counter()
            O.downsample(ds_clip[0], bits=10, quality=q, variant="avx2")
            res[f"downsample_q{q}"]["cpu_reference_ms_per_frame"] = round(
                1000 * (time.perf_counter() - t0), 1)
        res["cpu_reference"] = "reference AVX2 build (oracle/_ref), one host thread, one frame"
    sharpen.close()
    trecon.close()
    return res


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
FORMATS = {"420P8": S.YUV420P8, "420P10": S.YUV420P10, "420P16": S.YUV420P16,
           "420PS": S.YUV420PS, "422P10": S.YUV422P10, "444PS": S.YUV444PS}


def leg_specs(rank: int):
    """Frames of the timed legs beside the headline (each leg's frames are one
    batch): the 1080p algo 2 batch the batched-vs-per-frame target is stated
    on (the headline's 16 1080p frames, all run as algo 2), and the plain,
    jinc-resize and block-refinement configurations."""
    legs = {}
    legs["batched_1080p_p10_algo2"] = dict(
        reuse_headline=True, filter=dict(algo=2, **FILTER_ARGS),
        workload="16x1920x1080 YUV420P10 -> 4:4:4, algo 2, lanczos taps=4, sparse=1, qgate=1.0")
    legs["plain_720p_p8"] = dict(
        frames=[dict(width=1280, height=720, fmt="420P8", seed=R.frame_seed(8000, rank, i), gen={})
                for i in range(8)],
        filter=dict(algo=2, kernel="lanczos", taps=3, strength=0.8, sigma=0.01),
        workload="8x1280x720 YUV420P8 -> 4:4:4, algo 2, lanczos taps=3, strength 0.8, sigma 0.01")
    for fmt, tag in (("420P16", "p16"), ("420PS", "ps")):
        legs[f"jinc_resize_2160p_{tag}"] = dict(
            frames=[dict(width=1920, height=1080, fmt=fmt, seed=R.frame_seed(9000, rank, i),
                         gen={"antialias": True}) for i in range(12)],
            filter=dict(algo=4, kernel="jinc", taps=3, reg=0.005, width=3840, height=2160),
            workload=f"12x1920x1080 YUV{fmt} -> 3840x2160 4:4:4, jinc taps=3, algo 4, reg 0.005")
    legs["bm_bp_1080p_p8"] = dict(
        frames=[dict(width=1920, height=1080, fmt="420P8", seed=R.frame_seed(10000, rank, i),
                     gen={"extra_noise": True}) for i in range(16)],
        filter=dict(algo=2, bm=1, bp=1.0),
        workload="16x1920x1080 YUV420P8 (+noise) -> 4:4:4, algo 2, bm=1, bp=1.0")
    # where batching pays: frames too small to fill the GPU one at a time
    legs["small_frames_360p_algo2"] = dict(
        frames=[dict(width=640, height=360, fmt="420P10", seed=R.frame_seed(12000, rank, i), gen={})
                for i in range(64)],
        filter=dict(algo=2, **FILTER_ARGS),
        workload="64x640x360 YUV420P10 -> 4:4:4, algo 2, lanczos taps=4, sparse=1, qgate=1.0 "
                 "(not a reference configuration: the batched form's case)")
    return legs


def _gen_any(task):
    w, h, fmt, seed, gen = task
    return S.make_frame(w, h, FORMATS[fmt], seed=seed, **gen)


def generate_legs(legs, workers=None):
    tasks, owners = [], []
    for name, leg in legs.items():
        for k, fr in enumerate(leg.get("frames", [])):
            tasks.append((fr["width"], fr["height"], fr["fmt"], fr["seed"], fr["gen"]))
            owners.append((name, k))
    if not tasks:
        return {}
    workers = workers or min(len(tasks), max(1, (os.cpu_count() or 2) - 1), 16)
    with mp.get_context("spawn").Pool(workers) as pool:
        made = pool.map(_gen_any, tasks)
    out = {}
    for (name, k), planes in zip(owners, made):
        out.setdefault(name, []).append(planes)
    return out


def algorithmic_bytes(planes, out_w, out_h):
    """Compulsory HBM bytes of one frame: the input planes plus three output
    planes at the output sample size."""
    return sum(p.nbytes for p in planes) + 3 * out_w * out_h * planes[0].itemsize


def stage_frames(stage, kinds):
    """Indices of the frames a stage's launch processes; kinds[i] =
    (algo, guided, bm, bp, resize)."""
    def pick(fn):
        return [i for i, k in enumerate(kinds) if fn(*k)]
    if stage == "reconstructChroma":
        return pick(lambda a, g, bm, bp, rs: g and a in (2, 4))
    if stage.startswith(("buildAffineMaps", "buildDetail", "detailTransfer")):
        return pick(lambda a, g, bm, bp, rs: g and a == 6)
    if stage.startswith(("buildLGF", "blendSelector", "selector")):
        return pick(lambda a, g, bm, bp, rs: g and a == 4)
    if stage.startswith("collaborative"):
        return pick(lambda a, g, bm, bp, rs: bm)
    if stage.startswith("backProject"):
        return pick(lambda a, g, bm, bp, rs: bp)
    if stage.startswith("luma_resample"):
        return pick(lambda a, g, bm, bp, rs: rs)
    return list(range(len(kinds)))


lgcr = None       # the package, imported after the frame generators' spawn pools


class BatchLeg:
    """Frames resident in HBM, their filters, and the batched / per-frame
    device paths over them on one stream."""

    def __init__(self, lib, dev, stream, filters, planes_list):
        import numpy as np
        import torch
        self.lib, self.dev, self.stream = lib, dev, stream
        self.filters = filters
        self.dins, self.douts = [], []
        tdt = {np.uint8: torch.uint8, np.uint16: torch.int16, np.float32: torch.float32}
        for f, planes in zip(filters, planes_list):
            ins = []
            for p in planes:
                t = torch.from_numpy(p.view(np.int16) if p.dtype == np.uint16 else p).to(dev)
                ins.append(t.view(torch.uint16) if p.dtype == np.uint16 else t)
            self.dins.append(ins)
            odt = tdt[planes[0].dtype.type]
            outs = [torch.empty((f.out_h, f.out_w), dtype=odt, device=dev) for _ in range(3)]
            self.douts.append([o.view(torch.uint16) if odt == torch.int16 else o for o in outs])
        self.items = (lgcr.BatchItem * len(filters))()
        for i, f in enumerate(filters):
            self.items[i].filter = f.handle
            self.items[i].inp = lgcr.planes_desc(self.dins[i])
            self.items[i].out = lgcr.planes_desc(self.douts[i])
            self.items[i].chroma_location = -1
        self.batch = ctypes.c_void_p()
        assert lib.lgcr_batch_create(ctypes.byref(self.batch)) == 0
        self.out_pixels = sum(f.out_w * f.out_h for f in filters)
        self.algo_bytes = [algorithmic_bytes(p, f.out_w, f.out_h) for f, p in zip(filters, planes_list)]
        self.in_bytes = sum(sum(p.nbytes for p in planes) for planes in planes_list)

    def tune(self):
        """This batch's own autotuner (block shapes, guided variant, frame
        grouping) on its frames; untimed. Returns the report lines."""
        import torch
        rep = ctypes.create_string_buffer(8192)
        st = self.lib.lgcr_batch_autotune(self.batch, self.items, len(self.filters),
                                          ctypes.c_void_p(self.stream.cuda_stream), rep, 8192)
        torch.cuda.synchronize(self.dev)
        if st != 0:
            raise RuntimeError(self.lib.lgcr_last_error().decode())
        return [l for l in rep.value.decode().splitlines() if l]

    def run(self, use_graph=1):
        st = self.lib.lgcr_batch_run(self.batch, self.items, len(self.filters),
                                     ctypes.c_void_p(self.stream.cuda_stream), use_graph)
        if st != 0:
            raise RuntimeError(self.lib.lgcr_last_error().decode())

    def timed(self, fn, steps):
        import torch
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(self.stream)
        for _ in range(steps):
            fn()
        b.record(self.stream)
        torch.cuda.synchronize(self.dev)
        return a.elapsed_time(b)

    def per_frame(self):
        for i, f in enumerate(self.filters):
            f.frame(self.dins[i], -1, out=self.douts[i], stream=self.stream.cuda_stream)

    def stage_split(self, steps):
        """Per-stage device ms per step from event-bracketed runs (a separate
        pass: the bracketing bypasses the graph)."""
        lib = self.lib
        n = lib.lgcr_stage_count()
        lib.lgcr_batch_set_profiling(self.batch, 1)
        self.run(0)
        lib.lgcr_batch_stage_times(self.batch, None, None, 1)
        for _ in range(steps):
            self.run(0)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int * n)()
        lib.lgcr_batch_stage_times(self.batch, ms, cnt, 1)
        lib.lgcr_batch_set_profiling(self.batch, 0)
        return {lib.lgcr_stage_name(i).decode(): ms[i] / steps for i in range(n) if cnt[i]}

    def sparse_active(self):
        """Sparse-active ratio (trust-mask coverage) and active guided output
        pixels per frame, from one untimed per-frame pass with stats."""
        ratios, active = [], []
        for i, f in enumerate(self.filters):
            _, st = f.frame(self.dins[i], -1, out=self.douts[i], stream=self.stream.cuda_stream,
                            stats=True)
            ratios.append(st.sparse_active_ratio)
            active.append(int(st.active_output_pixels))
        return ratios, active

    def close(self):
        self.lib.lgcr_batch_destroy(self.batch)


def axis_active_means(f):
    """Mean active taps per output column and per output row of a filter's
    chroma axes (the reference's tap metric counts activeX * activeY per
    guided pixel, recon.cpp:253-257)."""
    import numpy as np
    lib = lgcr.library()
    lib.lgcr_debug_axis.restype = ctypes.c_int
    means = []
    for axis, n in ((0, f.out_w), (1, f.out_h)):
        shift = ctypes.c_double(-0.5 if axis == 0 else 0.0)
        sup = ctypes.c_int()
        lib.lgcr_debug_axis(f.handle, axis, shift, None, None, None, None, None, None, None,
                            None, None, ctypes.byref(sup))
        am = np.zeros(n * sup.value, np.uint8)
        lib.lgcr_debug_axis(f.handle, axis, shift, None, None, am.ctypes.data_as(ctypes.c_void_p),
                            None, None, None, None, None, None, ctypes.byref(sup))
        means.append(float(am.reshape(n, sup.value).sum(1).mean()))
    return means


# FP32 arithmetic of one guided tap (tapsSeparable in kernels_recon.cu): 27
# FP32 FLOPs (an FMA counted as 2) and 2 reciprocal approximations; with a
# jinc phase table the base weight is read instead of formed as wx * wy (26).
GUIDED_FP32_FLOP_PER_TAP = 27
GUIDED_FP32_FLOP_PER_RADIAL_TAP = 26
FP32_LANES_PER_SM, B200_SMS = 128, 148


def guided_fp32(rl, filt, active, kinds, sm_mhz):
    """When the dominant stage is the guided pass, add its counted FP32 work
    against the nominal FP32 rate: taps = active guided pixels x mean active
    taps per column x per row (the reference's tap metric, recon.cpp:253-257)."""
    if not rl or rl["kernel"] != "reconstructChroma":
        return
    mx, my = axis_active_means(filt)
    guided = stage_frames("reconstructChroma", kinds)
    taps = sum(active[i] for i in guided) * mx * my
    per_tap = GUIDED_FP32_FLOP_PER_RADIAL_TAP if filt.radial else GUIDED_FP32_FLOP_PER_TAP
    fp32_peak = B200_SMS * FP32_LANES_PER_SM * 2 * (sm_mhz or 1965.0) * 1e6 / 1e12
    achieved_tf = taps * per_tap / (rl["launch_ms"] / 1000.0) / 1e12
    rl["binding_bound"] = ("instruction issue and load latency of the FP32 (packed pairs), "
                           "FP64 accumulation and reciprocal pipes")
    rl["fp32"] = {"achieved_tflops": round(achieved_tf, 2), "peak_tflops": round(fp32_peak, 1),
                  "frac": round(achieved_tf / fp32_peak, 4),
                  "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 FLOP x sampled SM clock",
                  "taps_per_step": int(taps),
                  "taps_source": "active guided pixels x mean active taps per column x per row",
                  "flop_per_tap": per_tap}


def link_bandwidth(dev, nbytes=256 << 20, reps=3):
    """Host<->device copy rates of this box (pinned host memory, one large
    copy per direction, CUDA events): H2D alone, D2H alone, and both at once
    on two streams (the e2e leg's situation). GB/s; the e2e leg's copy
    roofline is its per-step bytes over these rates."""
    import torch
    h_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_in = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d_out = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    s1, s2 = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

    def run(h2d, d2h):
        start = torch.cuda.Event(enable_timing=True)
        ends = []
        start.record(s1)
        s2.wait_event(start)
        for on, stream, fn in ((h2d, s1, lambda: d_in.copy_(h_in, non_blocking=True)),
                               (d2h, s2, lambda: h_out.copy_(d_out, non_blocking=True))):
            if not on:
                continue
            with torch.cuda.stream(stream):
                for _ in range(reps):
                    fn()
                e = torch.cuda.Event(enable_timing=True)
                e.record(stream)
                ends.append(e)
        torch.cuda.synchronize(dev)
        return max(start.elapsed_time(e) for e in ends) / 1000.0

    run(True, True)                                   # warm-up
    gb = nbytes * reps / 1e9
    h2d = gb / run(True, False)
    d2h = gb / run(False, True)
    both = run(True, True)
    return {"h2d_gbs": round(h2d, 1), "d2h_gbs": round(d2h, 1),
            "duplex_gbs_each": round(gb / both, 1)}


def roofline_of(stage_ms, kinds, algo_bytes, peaks, steps_note):
    """Dominant stage: achieved algorithmic GB/s over the frames its launch
    processes vs the measured HBM copy bandwidth."""
    if not stage_ms:
        return None
    dominant = max(stage_ms, key=stage_ms.get)
    frames = stage_frames(dominant, kinds)
    launch_ms = stage_ms[dominant]
    nbytes = sum(algo_bytes[i] for i in frames)
    achieved = nbytes / (launch_ms / 1000.0) / 1e9
    peak = peaks.get("hbm_gbs", 6650.0)
    step_ms = sum(stage_ms.values())
    return {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "launch_ms": round(launch_ms, 3), "frames_in_launch": len(frames),
            "algorithmic_bytes_per_launch": int(nbytes),
            "step_hbm_frac": round(sum(algo_bytes) / (step_ms / 1000.0) / 1e9 / peak, 4),
            "stage_ms_per_step": {k: round(v, 3) for k, v in
                                  sorted(stage_ms.items(), key=lambda kv: -kv[1])},
            "stage_timing": steps_note}


def leg_only(args):
    """Profiler captures: run one leg alone (a configuration's batch, or the
    Sharpen / TRecon / Downsample clips; "filters" prints all three) for
    `steps` graph replays after `warmup` and print its time and stage
    split."""
    global lgcr
    rank = 0
    filter_legs = ("sharpen", "trecon", "downsample_q0", "downsample_q1", "downsample_q2", "filters")
    if args.leg in filter_legs:
        with mp.get_context("spawn").Pool(1) as pool:
            clip = pool.map(_gen_clip, [(R.frame_seed(11000, rank, 0), FILTERS_CLIP)])[0]
    else:
        legs = leg_specs(rank)
        if args.leg not in legs:
            raise SystemExit(f"unknown leg {args.leg!r}; one of {sorted(legs)} or {filter_legs}")
        leg = legs[args.leg]
        if leg.get("reuse_headline"):
            specs = [s for s in frame_specs(rank, args.frames) if s["width"] == 1920]
            planes_list = generate(specs)
        else:
            planes_list = generate_legs({args.leg: leg})[args.leg]
    import torch
    import lgcr as _lgcr
    lgcr = _lgcr
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    lib = lgcr.library()
    lib.lgcr_batch_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.lgcr_batch_stage_times.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    lib.lgcr_stage_name.restype = ctypes.c_char_p
    if args.leg in filter_legs:
        res = filters_leg(clip, dev, stream, args.steps, args.warmup)
        print(json.dumps({"leg": args.leg, **(res if args.leg == "filters" else res[args.leg])}))
        return 0
    if args.leg_frames > 0:
        planes_list = planes_list[:args.leg_frames]
    filters = [lgcr.Recon(lgcr.format_of(p, 10 if leg.get("reuse_headline") else None),
                          **leg["filter"]) for p in planes_list]
    b = BatchLeg(lib, dev, stream, filters, planes_list)
    tuned = [] if args.no_autotune else b.tune()
    for _ in range(max(args.warmup, 1)):
        b.run(1)
    torch.cuda.synchronize(dev)
    ms = b.timed(lambda: b.run(1), args.steps)
    b.per_frame()
    pms = b.timed(b.per_frame, args.steps)
    stage_ms = b.stage_split(1)
    b.close()
    print(json.dumps({"leg": args.leg, "frames": len(filters), "autotune": tuned,
                      "ms_per_step": round(ms / args.steps, 3),
                      "per_frame_ms_per_step": round(pms / args.steps, 3),
                      "mpix_s": round(b.out_pixels * args.steps / (ms / 1000) / 1e6, 1),
                      "stage_ms_per_step": {k: round(v, 3) for k, v in
                                            sorted(stage_ms.items(), key=lambda kv: -kv[1])}}))
    return 0


def our_arm(args):
    global lgcr
    rank, world, local = R.rank_info()
    specs = frame_specs(rank, args.frames)
    frames = generate(specs)                      # before CUDA init (spawn pools)
    legs = leg_specs(rank) if not args.no_legs else {}
    leg_frames = generate_legs(legs)
    clip = None
    if not args.no_legs:
        with mp.get_context("spawn").Pool(1) as pool:
            clip = pool.map(_gen_clip, [(R.frame_seed(11000, rank, 0), FILTERS_CLIP)])[0]
    cpu_frames = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu_frames = frames

    import numpy as np
    import torch
    import lgcr as _lgcr
    lgcr = _lgcr
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lib = lgcr.library()
    lib.lgcr_batch_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.lgcr_batch_stage_times.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    lib.lgcr_stage_name.restype = ctypes.c_char_p
    peaks = measured_peaks()
    stream = torch.cuda.Stream(device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()

    # filters (one per geometry x algo) and the headline batch, resident in HBM
    filt = {}
    for spec in specs:
        key = (spec["width"], spec["height"], spec["algo"])
        if key not in filt:
            fmt = lgcr.video_format(spec["width"], spec["height"], 10, 1, 1)
            filt[key] = lgcr.Recon(fmt, algo=spec["algo"], **FILTER_ARGS)
    head_filters = [filt[(s["width"], s["height"], s["algo"])] for s in specs]
    head = BatchLeg(lib, dev, stream, head_filters, frames)
    out_pixels = head.out_pixels

    # autotune launch shapes / register budget on this workload (untimed)
    tuned = ""
    if not args.no_autotune:
        rep = ctypes.create_string_buffer(4096)
        if lib.lgcr_autotune(head.items, len(specs), ctypes.c_void_p(stream.cuda_stream), rep, 4096) == 0:
            tuned = rep.value.decode()
        torch.cuda.synchronize(dev)
        # then the headline batch's own settings (frame grouping included)
        tuned += "\n".join("batch " + l for l in head.tune())

    # warm-up (tables, workspaces, the graphs of this layout)
    for _ in range(max(args.warmup, 1)):
        head.run(1)
    barrier()

    # timed region: batched form, graph replay, stage profiling off
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        start.record(stream)
        for _ in range(args.steps):
            head.run(1)
        stop.record(stream)
        barrier()
    elapsed_ms = start.elapsed_time(stop)
    launches_per_step = lib.lgcr_batch_launch_count(head.batch)
    max_ms = R.max_over_ranks(elapsed_ms, dev)
    value = out_pixels * world * args.steps / (max_ms / 1000.0) / 1e6
    clocks = clk.summary()

    # stage split from a separate event-bracketed pass (not the timed region)
    prof_steps = max(2, min(args.steps, 5))
    stage_ms = head.stage_split(prof_steps)
    barrier()
    if args.batch_only:
        head.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(value, 2), "unit": "Mpix/s",
                              "frames_per_step": len(specs), "batch_only": True,
                              "ms_per_step": round(max_ms / args.steps, 3),
                              "stage_ms_per_step": {k: round(v, 3) for k, v in
                                                    sorted(stage_ms.items(), key=lambda kv: -kv[1])}}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    # direct launches (no graph) of the same batch, for comparison
    head.run(0)
    direct_ms = head.timed(lambda: head.run(0), args.steps)
    # per-frame device path: one lgcr_recon_frame per frame on one stream
    head.per_frame()
    per_frame_ms = head.timed(head.per_frame, args.steps)
    barrier()
    ratios, active = head.sparse_active()

    # e2e: host planes in pinned memory through the per-frame C ABI, one host
    # thread per core (frame-parallel like the reference's fmParallel)
    pinned_in = []
    pinned_out = []
    for spec, planes in zip(specs, frames):
        ins = []
        for p in planes:
            t = torch.empty(p.shape, dtype=torch.int16, pin_memory=True)
            t.numpy()[...] = p.view(np.int16)
            ins.append(t.numpy().view(np.uint16))
        pinned_in.append(ins)
        outs = [None] + [torch.empty((spec["height"], spec["width"]), dtype=torch.int16,
                                     pin_memory=True).numpy().view(np.uint16) for _ in range(2)]
        pinned_out.append(outs)
    latencies = []

    e2e_threads = args.e2e_threads or min(16, cpu_threads())

    def e2e_pass(rounds=1, nthreads=e2e_threads, ins=pinned_in, outs=pinned_out):
        frame_queue(len(specs), rounds, nthreads,
                    lambda i: head_filters[i].frame(ins[i], -1, out=outs[i]), latencies)

    # untimed passes grow the per-filter workspace pools to the concurrency
    # the threads reach, so the timed passes allocate nothing
    e2e_pass(max(args.warmup, 1))
    latencies.clear()
    barrier()
    t0 = time.perf_counter()
    e2e_pass(args.steps)
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    e2e_s = R.max_over_ranks(e2e_s, dev)
    e2e_value = out_pixels * world * args.steps / e2e_s / 1e6
    e2e_latencies = list(latencies)
    # the same through pageable host buffers (how a VapourSynth host holds its
    # frames): the library stages them in pinned memory of its own
    page_in = [[np.array(p) for p in planes] for planes in frames]
    page_out = [[None] + [np.empty((s["height"], s["width"]), np.uint16) for _ in range(2)]
                for s in specs]
    e2e_pass(ins=page_in, outs=page_out)
    barrier()
    t0 = time.perf_counter()
    e2e_pass(args.steps, ins=page_in, outs=page_out)
    torch.cuda.synchronize(dev)
    e2e_page_s = R.max_over_ranks(time.perf_counter() - t0, dev)
    latencies[:] = e2e_latencies
    out_bytes_e2e = sum(2 * s["width"] * s["height"] * 2 for s in specs)   # U, V (luma shared)
    # copy roofline of the e2e leg: its bytes per step over the measured
    # duplex copy rate (both directions run at once)
    link = link_bandwidth(dev)
    copy_s = max(head.in_bytes, out_bytes_e2e) / (link["duplex_gbs_each"] * 1e9)
    link["copy_bound_mpix_s"] = round(out_pixels * world / copy_s / 1e6, 1)
    link["e2e_frac_of_copy_bound"] = round(e2e_value / link["copy_bound_mpix_s"], 3)

    # roofline of the dominant stage, with the guided stage's FP32 side
    kinds = [(s["algo"], True, False, False, False) for s in specs]
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    rl = roofline_of(stage_ms, kinds, head.algo_bytes, peaks,
                     f"event-bracketed pass of {prof_steps} steps")
    guided_fp32(rl, head_filters[0], active, kinds, sm_mhz)

    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded polygon frames)",
        "config": {"workload": WORKLOAD, "frames_per_step": len(specs),
                   "output_mpix_per_step": round(out_pixels / 1e6, 3),
                   "l2": "inputs larger than L2: ~250 MB in + 1 GB out per step",
                   "accumulation": "f32 with f64 accumulators (as the reference)",
                   "path": "batched form, CUDA graph replay, stage profiling off",
                   "parallelism": f"replicas x{world}",
                   "autotune": [l for l in tuned.splitlines() if l]},
        "sparse_active_ratio": {"mean": round(float(np.mean(ratios)), 4),
                                "min": round(float(np.min(ratios)), 4),
                                "max": round(float(np.max(ratios)), 4)},
        "per_frame": {"value": round(out_pixels * args.steps / (per_frame_ms / 1000) / 1e6, 2),
                      "unit": "Mpix/s", "ms_per_step": round(per_frame_ms / args.steps, 3)},
        "direct_launches": {"value": round(out_pixels * args.steps / (direct_ms / 1000) / 1e6, 2),
                            "unit": "Mpix/s", "ms_per_step": round(direct_ms / args.steps, 3)},
        "batched_vs_per_frame": round(per_frame_ms / max(elapsed_ms, 1e-9), 3),
        "latency_ms": {"p50": round(statistics.median(latencies), 3) if latencies else None,
                       "p99": round(sorted(latencies)[int(0.99 * (len(latencies) - 1))], 3)
                       if latencies else None, "per": "frame, e2e host path"},
        "e2e": {"value": round(e2e_value, 2), "unit": "Mpix/s", "host_threads": e2e_threads,
                "h2d_bytes_per_step": int(head.in_bytes), "d2h_bytes_per_step": int(out_bytes_e2e),
                "copy_roofline": link},
        "e2e_pageable": {"value": round(out_pixels * world * args.steps / e2e_page_s / 1e6, 2),
                         "unit": "Mpix/s", "host_threads": e2e_threads,
                         "buffers": "pageable numpy planes, staged by the library"},
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": rl,
        "clocks": clocks,
    }
    head.close()

    # the other legs: batched (graph) vs per-frame, stage split, roofline
    if legs:
        out_legs = {}
        leg_steps = max(3, min(args.steps, 10))
        for name, leg in legs.items():
            if leg.get("reuse_headline"):
                planes_list = [frames[i] for i, s in enumerate(specs) if s["width"] == 1920]
            else:
                planes_list = leg_frames[name]
            lf = [lgcr.Recon(lgcr.format_of(p, 10 if leg.get("reuse_headline") else None),
                             **leg["filter"]) for p in planes_list]
            b = BatchLeg(lib, dev, stream, lf, planes_list)
            leg_tuned = [] if args.no_autotune else b.tune()
            for _ in range(max(args.warmup, 1)):
                b.run(1)
            barrier()
            bms = b.timed(lambda: b.run(1), leg_steps)
            b.per_frame()
            pms = b.timed(b.per_frame, leg_steps)
            sms = b.stage_split(2)
            lr, la = b.sparse_active()
            fa = leg["filter"]
            kinds = [(fa.get("algo", 2), fa.get("strength", 0.8) > 0, bool(fa.get("bm")),
                      fa.get("bp", 0.0) > 0, "width" in fa)] * len(lf)
            leg_rl = roofline_of(sms, kinds, b.algo_bytes, peaks, "event-bracketed pass of 2 steps")
            guided_fp32(leg_rl, lf[0], la, kinds, (clocks or {}).get("sm_mhz"))
            out_legs[name] = {
                "workload": leg["workload"], "frames": len(lf),
                "batched": {"value": round(b.out_pixels * leg_steps / (bms / 1000) / 1e6, 2),
                            "unit": "Mpix/s", "ms_per_step": round(bms / leg_steps, 3)},
                "per_frame": {"value": round(b.out_pixels * leg_steps / (pms / 1000) / 1e6, 2),
                              "unit": "Mpix/s", "ms_per_step": round(pms / leg_steps, 3)},
                "batched_vs_per_frame": round(pms / max(bms, 1e-9), 3),
                "sparse_active_ratio": round(float(np.mean(lr)), 4),
                "launches_per_step": lib.lgcr_batch_launch_count(b.batch),
                "autotune": leg_tuned,
                "roofline": leg_rl}
            b.close()
            del lf
        result["legs"] = out_legs

    if clip is not None:
        result["filters"] = filters_leg(clip, dev, stream, max(3, min(args.steps, 10)), args.warmup)
        result["reference_scene"] = reference_scene_leg(dev, stream)

    if rank == 0 and args.serve_requests > 0:
        # content of the serving stream (spawned workers: safe after CUDA init)
        keys = [(k, s) for k in range(len(SERVE_KINDS)) for s in range(SERVE_SEEDS)]
        with mp.get_context("spawn").Pool(min(len(keys), max(1, (os.cpu_count() or 2) - 1), 16)) as pool:
            made = pool.map(_gen_serve, [(k, 7000 + 97 * k + s) for k, s in keys])
        result["serving"] = serving_leg(dict(zip(keys, made)), args.serve_requests, lanes=args.serve_lanes)
    if rank == 0 and cpu_frames is not None:
        threads = cpu_threads()
        value_cpu, total_s, times = run_cpu(cpu_frames, specs, 1, 0, threads, threads,
                                            min_seconds=10.0)
        result["cpu_baseline"] = {
            "value": round(value_cpu, 3), "unit": "Mpix/s", "cores": threads, "kind": "reference",
            "sample": f"{len(times)} rounds of {threads} frames (alternating 1080p/4K, algo 2/6, "
                      f"one frame per thread) from the workload, reference AVX2 build "
                      f"(oracle/_ref), {total_s:.1f} s",
            **host_cpu(),
            "reference_scene": reference_scene_fps()}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--frames", type=int, default=32,
                    help="frames per step (< 32 only for profiler captures)")
    ap.add_argument("--e2e-threads", type=int, default=0,
                    help="host threads calling the per-frame C ABI in the e2e leg (frames in "
                         "flight); default: the host's cores, at most 16, as the reference arm")
    ap.add_argument("--serve-requests", type=int, default=4000,
                    help="requests of the serving leg (0 skips it)")
    ap.add_argument("--serve-lanes", type=int, default=2,
                    help="concurrent device batches of the serving leg")
    ap.add_argument("--batch-only", action="store_true",
                    help="time the batched form only (profiler captures)")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the batched-target and per-workload legs")
    ap.add_argument("--leg", default="",
                    help="run one leg alone (profiler captures): a configuration leg's "
                         "name, sharpen or trecon")
    ap.add_argument("--leg-frames", type=int, default=0,
                    help="with --leg: keep only the first N frames of the leg (small captures)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the replicas under torchrun
        return R.relaunch(os.path.abspath(__file__), sys.argv[1:], args.gpus)
    if args.impl == "reference":
        return reference_arm(args)
    if args.leg:
        return leg_only(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
