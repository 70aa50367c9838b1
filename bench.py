#!/usr/bin/env python
"""Benchmark of the B200 ISP: Gpix/s on one frame shape, bit-exact path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload c1]

A step is one frame through the ISP. The default workload is a 3840x2160
GRBG MIPI RAW10 frame with gray-world white balance, Malvar-He-Cutler
demosaic, sharpening 0.5, the colour matrix, a 1024-entry sRGB table, RGB16
output, histogram and statistics (the HBM-roofline frame shape). Frames are
independent, so N GPUs run N replicas on their own frames (weak scaling, no
collective on the data path); torch.distributed is used only for the barrier
and the max over ranks of the timed region.

`value` is device-resident throughput (inputs already in HBM, rotating over
buffer sets that together exceed L2), timed with CUDA events on the
launching stream. `e2e` is the same metric through the host-buffer C-ABI call
(isp_b200_process_host: host->device copy of the raw frame, the kernels, and
the device->host copy of the image, histogram and statistics, every step).
`roofline` is the fused tile kernel's compulsory bytes over its own
event-timed duration. `cpu_baseline` is the reference's CPU backend (built
from its sources into oracle/_ref) on the host cores, a bounded sample.

At one GPU the default c1 line also carries `batch` (c3: the 48-camera
mixed batch as one replayed graph per step against the same frames through
the per-frame path) and `serving` (c4, bounded: the 64 streams at their
nominal Poisson rates for the latency percentiles, then saturation runs
batched and per frame), so that both are measured on the same box under the
same clock; --no-extras leaves them out.

--impl reference times that CPU backend alone on the same workload and prints
the same line with "impl": "reference".

--workload convert measures the colour converter (the step after the ISP):
a 3840x2160 RGB8 frame into NV12 as the headline line, plus every case of
the reference converter's benchmark beside the reference's own CUDA kernel
(built from its sources into oracle/_ref) in a "cases" table.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "holoscan-zozo-modules_b200"))

import numpy as np  # noqa: E402

from isp_b200 import abi, scene  # noqa: E402

L2_BYTES = 126 * 1024 * 1024
METRIC = "ISP Gpix/s (bit-exact vs the reference CPU backend)"
WORKLOADS = {"c0": scene.config0, "c1": scene.config1, "c2": scene.config2}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["c3", "c4", "convert", "view"], default="c1")
    ap.add_argument("--seconds", type=float, default=60.0, help="c4: the nominal-rate serving run")
    ap.add_argument("--aux-seconds", type=float, default=15.0, help="c4: the other serving runs")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="c1 at one GPU: skip the batch and serving keys")
    ap.add_argument("--serving-seconds", type=float, default=20.0, help="c1's serving key: the nominal-rate run")
    ap.add_argument("--serving-sat-seconds", type=float, default=5.0, help="c1's serving key: each saturation run")
    ap.add_argument("--no-cases", action="store_true", help="convert: the headline case only")
    ap.add_argument("--fresh-frames", type=int, default=0,
                    help="c2: render this many fresh-seed frames instead of the workload's 200 (small profiling runs)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The largest of every rank's x (all_reduce MAX; x itself on one rank)."""
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, seconds: float, world: int, dist=None, device: str = "cuda") -> float:
    """Units all ranks processed over the slowest rank's time. Every rank does
    the same work (replicas, weak scaling), so the job's units are world x
    units_per_rank and it ends when its slowest rank does."""
    return world * units_per_rank / max_over_ranks(seconds, dist, device)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(kernel: str, workload: str):
    """dram bytes per launch of `kernel` from its committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1].strip()))
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi samples of the GPU's clocks and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---- CPU: the reference's own backend on the host cores ---------------------

def cpu_pipeline_factory():
    """The reference CPU backend (oracle/_ref) where built, else the C oracle."""
    import oracle

    if oracle.reference_available():
        return oracle.ReferencePipeline, "reference"
    return oracle.OraclePipeline, "port"


def cpu_threads() -> int:
    n = os.cpu_count() or 1
    try:
        import psutil

        n = min(n, max(1, int(psutil.virtual_memory().available // (400 * 1024 * 1024))))
    except ImportError:
        pass
    return max(1, min(n, 64))


def cpu_throughput(w: scene.Workload, raw: abi.RawFrame, seconds: float, threads: int):
    """Frames per second of `threads` independent CPU pipelines for about `seconds`."""
    make, kind = cpu_pipeline_factory()
    pipes = [make(w.params) for _ in range(threads)]
    for p in pipes[:1]:
        p.process(raw, w.out_format, w.with_stats)  # warm-up: first touches of the scratch
    counts = [0] * threads
    stop = time.perf_counter() + seconds

    def work(i):
        p = pipes[i]
        while time.perf_counter() < stop or counts[i] == 0:
            p.process(raw, w.out_format, w.with_stats)
            counts[i] += 1

    t0 = time.perf_counter()
    ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    elapsed = time.perf_counter() - t0
    frames = sum(counts)
    return frames, elapsed, kind


def crop_rows(raw: abi.RawFrame, rows: int) -> abi.RawFrame:
    """The first `rows` rows of a raw frame (rows are independent in every format)."""
    return abi.RawFrame(raw.data[: rows * raw.pitch], raw.width, rows, raw.pitch, raw.format, raw.bit_depth,
                        raw.pattern)


def run_reference(args):
    """The reference's CPU backend on the host cores: each step, every thread
    processes a band of the workload's frame, the band sized so that the
    whole run takes about a minute and a half whatever --steps and --warmup."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    w = WORKLOADS.get(args.workload, scene.config1)()
    raw = w.raw(1)
    threads = cpu_threads()
    make, kind = cpu_pipeline_factory()
    pipes = [make(w.params) for _ in range(threads)]

    def step(rows):
        band = crop_rows(raw, rows)
        t0 = time.perf_counter()
        ts = [threading.Thread(target=pipes[i].process, args=(band, w.out_format, w.with_stats)) for i in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    # Calibrate on a 64-row band, then size the band to the time budget.
    probe = min(64, w.height)
    step(probe)
    per_row = step(probe) / probe
    budget = min(3.0, max(0.05, 90.0 / (args.steps + args.warmup)))
    rows = int(budget / per_row) // 2 * 2
    rows = max(2, min(w.height, rows))
    step_times = []
    for i in range(args.warmup + args.steps):
        t = step(rows)
        if i >= args.warmup:
            step_times.append(t)
    total = sum(step_times)
    value = threads * w.width * rows * len(step_times) / total / 1e9
    sample = f"{threads} threads x a {w.width}x{rows} band of the {w.width}x{w.height} frame per step"
    line = {
        "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / len(step_times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
        "config": workload_config(w), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Gpix/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(w: scene.Workload):
    cfg = {"workload": w.name, "width": w.width, "height": w.height,
           "pattern": ["RGGB", "BGGR", "GRBG", "GBRG"][w.pattern], "raw_format": ["u8", "u16", "RAW10", "RAW12"][w.fmt],
           "bit_depth": w.bits, "output": ["RGB8", "RGBA8", "RGB16", "RGB32F"][w.out_format],
           "white_balance": ["manual", "gray-world", "white-patch"][w.params.white_balance],
           "demosaic": ["bilinear", "malvar"][w.params.demosaic], "sharpen": w.params.sharpen,
           # The reference's histogram output is [4][256] (luma, R, G, B of the
           # 8-bit codes of the stored image); it has no 1024-bin form.
           "histogram": "[4][256] of the 8-bit output codes" if w.with_hist else False,
           "stats": w.with_stats, "compulsory_bytes_per_frame": w.compulsory_bytes()}
    if w.fresh_frames:
        cfg["frames"] = (f"{w.fresh_frames} fresh-seed frames rendered on the device (isp_b200_synthetic_raw), "
                         f"taken in turn: {w.fresh_frames * abi.raw_row_bytes(w.fmt, w.width) * w.height / 1e9:.1f} GB "
                         "of raw, far above the 126 MB L2")
    else:
        # Both arms name the same workload; the GPU arm's inputs exceed L2.
        nbuf = rotating_sets(w)
        cfg["l2"] = (f"GPU arm: {nbuf} rotating buffer sets, {nbuf * w.compulsory_bytes() / 1e6:.0f} MB > 126 MB L2; "
                     "CPU arm: one frame")
    return cfg


def rotating_sets(w: scene.Workload) -> int:
    """Buffer sets the GPU arm rotates over, together above twice the L2."""
    return max(2, math.ceil(2 * L2_BYTES / w.compulsory_bytes()))


# ---- GPU ---------------------------------------------------------------------

def batch_summary(steps: int, warmup: int, barrier, clocks=None) -> dict:
    """c3 at one GPU for the default line's `batch` key: the 48-frame mixed
    batch replayed as a CUDA graph against the same frames through the
    per-frame path, device-resident inputs, CUDA-event timed."""
    core = batch_core(steps, warmup, 0, barrier, clocks)
    info = core["batch"].info()
    core["batch"].close()
    per_step = core["elapsed_ms"] / steps
    px = core["total_px"]
    return {"workload": "c3_mixed_batch_48_frames", "value": px / (per_step / 1e3) / 1e9, "unit": "Gpix/s",
            "ms_per_step": per_step, "steps": steps, "warmup": warmup, "pixels_per_step": px,
            "per_frame_path_value": px / (core["plain_ms"] / 1e3) / 1e9, "per_frame_path_ms_per_step": core["plain_ms"],
            "batched_over_per_frame": core["plain_ms"] / per_step,
            "launch": "descriptor staging + statistics pass + tile pass per step, replayed CUDA graph; per-frame "
                      "path: one isp_b200_process per frame on one stream",
            "autotune": info, "per_frame_tile_rows": core["per_frame_tile_rows"], "clocks": core["clocks"]}


def serving_summary(nominal_seconds: float, sat_seconds: float, barrier, clocks=None) -> dict:
    """c4 at one GPU for the default line's `serving` key, bounded: the 64
    streams at their nominal Poisson rates with host-memory arrivals for
    `nominal_seconds` (latency percentiles), then closed-loop saturation runs
    of `sat_seconds`, batched and per frame, with device-memory arrivals."""
    cams, fps, budget, serve, brief = serving_setup(0, barrier)
    nominal = serve(False, False, False, nominal_seconds, clocks)
    sat = serve(False, True, True, sat_seconds)
    sat_plain = serve(True, True, True, sat_seconds)
    ratio = sat["gpix_per_s"] / max(1e-9, sat_plain["gpix_per_s"])
    return {"workload": "c4_serving_64_streams", "unit": "Gpix/s",
            "latency_ms": {"p50": nominal["p50_ms"], "p99": nominal["p99_ms"], "p99.9": nominal["p999_ms"],
                           "max": nominal["max_ms"], "arrivals": "host memory (copied in), nominal rate",
                           "seconds": nominal_seconds},
            "nominal": brief(nominal), "offered_gpix_s": sum(c.pixels * f for c, f in zip(cams, fps)) / 1e9,
            "saturation_value": sat["gpix_per_s"], "saturation": brief(sat),
            "per_frame_path_value": sat_plain["gpix_per_s"], "per_frame_path": brief(sat_plain),
            "batched_over_per_frame": ratio, "saturation_seconds": sat_seconds, "memory_budget_bytes": budget,
            "targets": {"batched_at_least_2x_per_frame": ratio >= 2.0, "p99_at_most_1_ms": nominal["p99_ms"] <= 1.0},
            "clocks": nominal["clocks"]}


def run_b200(args):
    import torch

    import isp_b200

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    w = WORKLOADS[args.workload]()
    if args.fresh_frames > 0 and w.fresh_frames:
        w.fresh_frames = args.fresh_frames
    raw = w.raw(1 + rank)
    out_row = w.width * abi.output_channels(w.out_format) * abi.output_channel_bytes(w.out_format)
    nbuf = rotating_sets(w)
    if w.fresh_frames:
        # Fresh seeds: distinct frames rendered on the device, taken in turn.
        nraw = w.fresh_frames
        raws = []
        for i in range(nraw):
            buf = torch.empty(raw.pitch * w.height, dtype=torch.uint8, device="cuda")
            isp_b200.synthetic_raw(w.width, w.height, w.fmt, w.bits, w.pattern, w.black, 100_000 * (rank + 1) + i,
                                   buf.data_ptr(), raw.pitch)
            raws.append(buf)
        torch.cuda.synchronize()
    else:
        nraw = nbuf
        raws = [torch.from_numpy(raw.data).cuda() for _ in range(nbuf)]
    outs = [torch.empty(w.height * out_row, dtype=torch.uint8, device="cuda") for _ in range(nbuf)]
    hists = [torch.empty(1024, dtype=torch.int32, device="cuda") for _ in range(nbuf)]
    stats = [torch.empty(12, dtype=torch.float32, device="cuda") for _ in range(nbuf)]
    pipe = isp_b200.Pipeline(w.params)
    views = []
    for i in range(max(nraw, nbuf)):
        rv = abi.RawViewC(raws[i % nraw].data_ptr(), w.width, w.height, raw.pitch, w.fmt, w.bits, w.pattern)
        ov = abi.RgbViewC(outs[i % nbuf].data_ptr(), out_row, w.out_format)
        st = abi.StatsC(hists[i % nbuf].data_ptr() if w.with_hist else None,
                        stats[i % nbuf].data_ptr() if w.with_stats else None)
        views.append((rv, ov, st))
    exp = abi.ExposureC(10_000_000, 2.0)
    L = isp_b200.lib()
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)

    def step(i):
        rv, ov, st = views[i % len(views)]
        isp_b200.check(L.isp_b200_process(pipe.handle, C.byref(rv), C.byref(ov), C.byref(st), C.byref(exp), sptr))

    launches_per_step = 2 if w.params.white_balance != abi.MANUAL else 1
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        clocks = Clocks(local)
        clocks.start()
        time.sleep(0.3)
        barrier()
        start.record(stream)
        for i in range(args.steps):
            step(i)
        end.record(stream)
        barrier()
        clock_info = clocks.stop()
        # The fused tile kernel alone (the roofline's kernel): events recorded
        # around it in a second run of steps. They keep it from overlapping
        # the statistics pass, so this is its own duration.
        ksteps = min(args.steps, 400)
        before = [torch.cuda.Event(enable_timing=True) for _ in range(ksteps)]
        after = [torch.cuda.Event(enable_timing=True) for _ in range(ksteps)]
        for e in before + after:
            e.record(stream)  # creates the CUDA event behind the handle
        for i in range(ksteps):
            L.isp_b200_set_kernel_events(pipe.handle, C.c_void_p(before[i].cuda_event), C.c_void_p(after[i].cuda_event))
            step(i)
        L.isp_b200_set_kernel_events(pipe.handle, None, None)
        torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(end)
    kernel_ms = sum(b.elapsed_time(a) for b, a in zip(before, after)) / ksteps
    elapsed_max = max_over_ranks(elapsed_ms, dist)
    value = whole_job_rate(args.steps * w.pixels, elapsed_ms / 1e3, world, dist) / 1e9

    # End to end through the host-buffer call, pinned host memory, every step.
    e2e_steps = max(3, min(args.steps, 40))
    host_raw = torch.from_numpy(raw.data).pin_memory().numpy()
    host_raw_frame = abi.RawFrame(host_raw, w.width, w.height, raw.pitch, w.fmt, w.bits, w.pattern)
    host_out = torch.empty((w.height, out_row), dtype=torch.uint8).pin_memory().numpy()
    host_out_typed = host_out.view(abi.output_dtype(w.out_format)).reshape(w.height, w.width, abi.output_channels(w.out_format))
    for _ in range(3):
        pipe.process_host(host_raw_frame, w.out_format, w.with_stats, (10_000_000, 2.0), out=host_out_typed)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        pipe.process_host(host_raw_frame, w.out_format, w.with_stats, (10_000_000, 2.0), out=host_out_typed)
    e2e_s = time.perf_counter() - t0
    e2e_sync_value = whole_job_rate(e2e_steps * w.pixels, e2e_s, world, dist) / 1e9
    h2d = abi.raw_row_bytes(w.fmt, w.width) * w.height
    d2h = w.height * out_row + (4096 if w.with_hist else 0) + (48 if w.with_stats else 0)

    # Streamed, as a capture loop uses the public asynchronous call: every
    # frame is copied in from pinned host memory (upload stream), processed by
    # isp_b200_process (compute stream) and its image, histogram and
    # statistics copied back (download stream), three frames in flight, so
    # that one frame's upload overlaps another's download on the full-duplex
    # link. The timed region spans the first upload to the last download.
    nslot = 3
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    host_in = torch.from_numpy(raw.data).pin_memory()
    dev_in = [torch.empty_like(host_in, device="cuda") for _ in range(nslot)]
    dev_out = [torch.empty(w.height * out_row, dtype=torch.uint8, device="cuda") for _ in range(nslot)]
    dev_hist = [torch.empty(1024, dtype=torch.int32, device="cuda") for _ in range(nslot)]
    dev_st = [torch.empty(12, dtype=torch.float32, device="cuda") for _ in range(nslot)]
    host_o = [torch.empty(w.height * out_row, dtype=torch.uint8).pin_memory() for _ in range(nslot)]
    host_h = [torch.empty(1024, dtype=torch.int32).pin_memory() for _ in range(nslot)]
    host_s = [torch.empty(12, dtype=torch.float32).pin_memory() for _ in range(nslot)]
    ev_in = [torch.cuda.Event() for _ in range(nslot)]
    ev_done = [torch.cuda.Event() for _ in range(nslot)]
    ev_out = [torch.cuda.Event() for _ in range(nslot)]
    slot_views = []
    for k in range(nslot):
        rv = abi.RawViewC(dev_in[k].data_ptr(), w.width, w.height, raw.pitch, w.fmt, w.bits, w.pattern)
        ov = abi.RgbViewC(dev_out[k].data_ptr(), out_row, w.out_format)
        st = abi.StatsC(dev_hist[k].data_ptr() if w.with_hist else None, dev_st[k].data_ptr() if w.with_stats else None)
        slot_views.append((rv, ov, st))

    def streamed(i):
        k = i % nslot
        if i >= nslot:
            up.wait_event(ev_out[k])  # the slot's previous frame is back on the host
        with torch.cuda.stream(up):
            dev_in[k].copy_(host_in, non_blocking=True)
        ev_in[k].record(up)
        stream.wait_event(ev_in[k])
        rv, ov, st = slot_views[k]
        isp_b200.check(L.isp_b200_process(pipe.handle, C.byref(rv), C.byref(ov), C.byref(st), C.byref(exp), sptr))
        ev_done[k].record(stream)
        down.wait_event(ev_done[k])
        with torch.cuda.stream(down):
            host_o[k].copy_(dev_out[k], non_blocking=True)
            if w.with_hist:
                host_h[k].copy_(dev_hist[k], non_blocking=True)
            if w.with_stats:
                host_s[k].copy_(dev_st[k], non_blocking=True)
        ev_out[k].record(down)

    stream_steps = max(3 * nslot, min(args.steps, 60))
    for i in range(nslot):
        streamed(i)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for i in range(stream_steps):
        streamed(i)
    torch.cuda.synchronize()
    e2e_stream_s = time.perf_counter() - t0
    e2e_value = whole_job_rate(stream_steps * w.pixels, e2e_stream_s, world, dist) / 1e9

    # The reference's own CUDA backend for sm_100a on the same device frames,
    # stream and step, after the timed region (the GPU bar; not this build).
    ref_gpu = None
    if rank == 0 and world == 1:
        import oracle

        if oracle.reference_cuda_available():
            rp = oracle.ReferenceCudaPipeline(w.params)
            rsteps = min(args.steps, 400)
            with torch.cuda.stream(stream):
                for i in range(10):
                    rv, ov, st = views[i % len(views)]
                    rp.process(rv, ov, st, exp, stream.cuda_stream)
                ra, rb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ra.record(stream)
                for i in range(rsteps):
                    rv, ov, st = views[i % len(views)]
                    rp.process(rv, ov, st, exp, stream.cuda_stream)
                rb.record(stream)
                rb.synchronize()
            rms = ra.elapsed_time(rb) / rsteps
            # One frame from each, byte for byte (informational).
            rv, ov, st = views[0]
            torch.cuda.synchronize()
            rp.close()
            pipe.reset()
            rp2 = oracle.ReferenceCudaPipeline(w.params)
            rp2.process(rv, ov, st, exp, 0)
            torch.cuda.synchronize()
            theirs = outs[0].cpu().numpy().copy()
            rp2.close()
            isp_b200.check(L.isp_b200_process(pipe.handle, C.byref(rv), C.byref(ov), C.byref(st), C.byref(exp), None))
            torch.cuda.synchronize()
            same = bool(np.array_equal(theirs, outs[0].cpu().numpy()))
            ref_gpu = {"value": w.pixels / (rms / 1e3) / 1e9, "unit": "Gpix/s", "ms_per_step": rms, "steps": rsteps,
                       "speedup_of_this_build": (rms / 1e3) / (elapsed_ms / 1e3 / args.steps),
                       "image_bytes_equal": same,
                       "library": "oracle/_ref/libisp_ref_cuda.so (the reference's cuda_pipeline.cu, sm_100a, "
                                  "--fmad=false)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        frames, secs, kind = cpu_throughput(w, raw, args.cpu_seconds, threads)
        cpu = {"value": frames * w.pixels / secs / 1e9, "unit": "Gpix/s", "cores": threads, "kind": kind,
               "sample": f"{frames} frames of {w.width}x{w.height} over {secs:.1f} s on {threads} threads"}
        # One thread, the mean of 5 frames after 1 warm-up, as the reference's
        # benchmark times its CPU backend (modules/isp/tests/benchmark.cpp:147-165).
        make, _ = cpu_pipeline_factory()
        single = make(w.params)
        single.process(raw, w.out_format, w.with_stats)
        t0 = time.perf_counter()
        for _ in range(5):
            single.process(raw, w.out_format, w.with_stats)
        per_frame = (time.perf_counter() - t0) / 5
        cpu["single_thread"] = {"value": w.pixels / per_frame / 1e9, "unit": "Gpix/s", "ms_per_frame": per_frame * 1e3,
                                "sample": "1 thread, mean of 5 frames after 1 warm-up"}

    if dist is not None:
        dist.barrier()
    pipe.close()

    # c3 and c4 beside c1 at one GPU (the default run): the batched launch
    # and the serving loop on the same box, under the same clock.
    extras = {}
    if world == 1 and args.workload == "c1" and not args.no_extras:
        extras["batch"] = batch_summary(max(20, min(args.steps, 200)), max(3, args.warmup), barrier, Clocks(local))
        extras["serving"] = serving_summary(args.serving_seconds, args.serving_sat_seconds, barrier, Clocks(local))
    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = w.compulsory_bytes() / (kernel_ms / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "config": workload_config(w),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic("isp_main_kernel", args.workload),
                         "kernel": "isp_main_kernel", "kernel_ms": kernel_ms, "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gpix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": stream_steps,
                    "api": "isp_b200_process with pinned-host uploads and downloads on their own streams, "
                           "three frames in flight",
                    "synchronous_value": e2e_sync_value,
                    "synchronous_api": "isp_b200_process_host (one frame at a time, copies not overlapped)"},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clock_info,
            "reference_gpu": ref_gpu,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def batch_core(steps: int, warmup: int, rank: int, barrier, clocks=None) -> dict:
    """c3's timed core: the 48 cameras' device-rendered frames through the
    batch (autotuned, replayed CUDA graph) for `steps` launches after
    `warmup`, then the same frames through the per-frame path (one
    isp_b200_process each). Times are CUDA events on the launching stream."""
    import torch

    import isp_b200

    cams = scene.mixed_cameras(seed=2024)
    pipes = [isp_b200.Pipeline(c.params) for c in cams]
    frames = []
    for i, c in enumerate(cams):
        data, row = device_frame(c, 7000 * (rank + 1) + i)
        out_row = c.width * 3
        out = torch.empty(c.height * out_row, dtype=torch.uint8, device="cuda")
        hist = torch.empty(1024, dtype=torch.int32, device="cuda")
        st = torch.empty(12, dtype=torch.float32, device="cuda")
        rv = abi.RawViewC(data.data_ptr(), c.width, c.height, row, c.fmt, c.bits, c.pattern)
        ov = abi.RgbViewC(out.data_ptr(), out_row, abi.RGB8)
        frames.append((data, out, hist, st, rv, ov, row, out_row))
    total_px = sum(c.pixels for c in cams)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    # The per-frame path's tile height per camera shape (isp_b200_autotune on
    # the first camera of each shape), applied to every camera of the shape.
    picks = {}
    for i, c in enumerate(cams):
        key = f"{c.width}x{c.height} {['u8', 'u16', 'RAW10', 'RAW12'][c.fmt]}/{c.bits}"
        if key not in picks:
            data, out, hist, st, rv, ov, row, out_row = frames[i]
            picks[key] = pipes[i].autotune(rv, ov, hist.data_ptr(), st.data_ptr(), (10_000_000, 1.5), sptr)
        pipes[i].set_tile_rows(picks[key])
    batch = isp_b200.Batch(len(cams))
    for pipe, (data, out, hist, st, rv, ov, row, out_row) in zip(pipes, frames):
        batch.add(pipe, rv, ov, hist.data_ptr(), st.data_ptr(), (10_000_000, 1.5))
    batch.autotune(sptr)
    for _ in range(warmup):
        batch.launch(sptr, True)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    if clocks is not None:
        clocks.start()
    time.sleep(0.3)
    barrier()
    start.record(stream)
    for _ in range(steps):
        batch.launch(sptr, True)
    end.record(stream)
    barrier()
    clock_info = clocks.stop() if clocks is not None else None
    elapsed_ms = start.elapsed_time(end)
    # The same frames through the per-frame path (one isp_b200_process each).
    for _ in range(2):
        for pipe, (data, out, hist, st, rv, ov, row, out_row) in zip(pipes, frames):
            pipe.process(rv, ov, hist.data_ptr(), st.data_ptr(), (10_000_000, 1.5), sptr)
    p_start, p_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain_steps = max(3, steps // 2)
    barrier()
    p_start.record(stream)
    for _ in range(plain_steps):
        for pipe, (data, out, hist, st, rv, ov, row, out_row) in zip(pipes, frames):
            pipe.process(rv, ov, hist.data_ptr(), st.data_ptr(), (10_000_000, 1.5), sptr)
    p_end.record(stream)
    barrier()
    plain_ms = p_start.elapsed_time(p_end) / plain_steps
    return {"cams": cams, "pipes": pipes, "frames": frames, "batch": batch, "stream": stream, "total_px": total_px,
            "elapsed_ms": elapsed_ms, "plain_ms": plain_ms, "clocks": clock_info, "per_frame_tile_rows": picks}


def run_batch(args):
    """The mixed batch: 48 cameras' frames of four shapes through one launch
    per pass (a replayed CUDA graph), against the same frames through the
    per-frame path."""
    import torch

    import isp_b200

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    core = batch_core(args.steps, args.warmup, rank, barrier, Clocks(local))
    cams, pipes, frames, batch, stream = core["cams"], core["pipes"], core["frames"], core["batch"], core["stream"]
    sptr = stream.cuda_stream
    total_px, elapsed_ms, plain_ms, clock_info = core["total_px"], core["elapsed_ms"], core["plain_ms"], core["clocks"]
    elapsed_max = max_over_ranks(elapsed_ms, dist)
    value = whole_job_rate(args.steps * total_px, elapsed_ms / 1e3, world, dist) / 1e9
    # End to end: every step copies each frame's raw from pinned host memory,
    # runs the batch, and copies each image, histogram and statistics back.
    # Two buffer sets alternate so that one step's uploads (upload stream)
    # overlap the previous step's downloads (download stream) on the
    # full-duplex link; the cameras' frames stay in order on the compute stream.
    host_in = [torch.empty(f[0].numel(), dtype=torch.uint8).pin_memory() for f in frames]
    for h, f in zip(host_in, frames):
        h.copy_(f[0])
    second = []
    for c, f in zip(cams, frames):
        data2 = torch.empty_like(f[0])
        out2 = torch.empty_like(f[1])
        hist2 = torch.empty_like(f[2])
        st2 = torch.empty_like(f[3])
        rv2 = abi.RawViewC(data2.data_ptr(), c.width, c.height, f[6], c.fmt, c.bits, c.pattern)
        ov2 = abi.RgbViewC(out2.data_ptr(), f[7], abi.RGB8)
        second.append((data2, out2, hist2, st2, rv2, ov2, f[6], f[7]))
    sets = [frames, second]
    host_out = [[torch.empty(f[1].numel(), dtype=torch.uint8).pin_memory() for f in frames] for _ in range(2)]
    host_st = [[torch.empty(1024 + 12, dtype=torch.int32).pin_memory() for _ in frames] for _ in range(2)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    e2e_steps = max(4, min(args.steps, 12))

    def e2e_step(i):
        k = i % 2
        if i >= 2:
            up.wait_event(ev_out[k])  # this set's previous results are back on the host
        with torch.cuda.stream(up):
            for h, f in zip(host_in, sets[k]):
                f[0].copy_(h, non_blocking=True)
        ev_in[k].record(up)
        stream.wait_event(ev_in[k])
        batch.clear()
        for pipe, f in zip(pipes, sets[k]):
            batch.add(pipe, f[4], f[5], f[2].data_ptr(), f[3].data_ptr(), (10_000_000, 1.5))
        batch.launch(sptr, True)
        ev_done[k].record(stream)
        down.wait_event(ev_done[k])
        with torch.cuda.stream(down):
            for h, hs, f in zip(host_out[k], host_st[k], sets[k]):
                h.copy_(f[1], non_blocking=True)
                hs[:1024].copy_(f[2], non_blocking=True)
                hs[1024:].copy_(f[3].view(torch.int32), non_blocking=True)
        ev_out[k].record(down)

    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        e2e_step(i)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = whole_job_rate(e2e_steps * total_px, e2e_s, world, dist) / 1e9
    h2d = sum(f[0].numel() for f in frames)
    d2h = sum(f[1].numel() + 4096 + 48 for f in frames)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_mixed_baseline(cams, (0, 16, 32, 44), args.cpu_seconds)
    info = batch.info()
    batch.close()
    if rank == 0:
        peak, peak_kind = measured_peak()
        compulsory = sum(abi.raw_row_bytes(c.fmt, c.width) * c.height + c.pixels * 3 for c in cams)
        achieved = compulsory / (elapsed_max / args.steps / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "config": {"workload": "c3_mixed_batch_48_frames", "frames": len(cams), "pixels_per_step": total_px,
                       "shapes": "16x640x480 u8 RGGB, 16x1920x1080 u16/12 GBRG, 12x3840x2160 RAW10 GRBG, "
                                 "4x4096x3072 u16/16 BGGR", "output": "RGB8", "histogram": True, "stats": True,
                       "launch": "descriptor staging + one statistics pass + one tile pass per step, replayed CUDA graph",
                       "per_frame_path_gpix_s": total_px / (plain_ms / 1e3) / 1e9,
                       "per_frame_path_ms_per_step": plain_ms, "batch_over_per_frame": plain_ms / (elapsed_max / args.steps),
                       "autotune": info, "per_frame_tile_rows": core["per_frame_tile_rows"],
                       "l2": f"inputs + outputs {compulsory / 1e6:.0f} MB > 126 MB L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "batch step (statistics + tile passes)", "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gpix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps,
                    "api": "isp_b200_batch_launch with per-frame host copies, two buffer sets: uploads overlap the "
                           "previous step's downloads"},
            "gpu_launches": 3 * args.steps, "clocks": clock_info,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def device_frame(c, seed: int):
    """Camera c's frame of `seed`, rendered on the device by isp_b200_synthetic_raw:
    a uint8 tensor of rows and the row bytes."""
    import torch

    import isp_b200

    row = abi.raw_row_bytes(c.fmt, c.width)
    data = torch.empty(row * c.height, dtype=torch.uint8, device="cuda")
    isp_b200.synthetic_raw(c.width, c.height, c.fmt, c.bits, c.pattern, c.black, seed, data.data_ptr(), row)
    return data, row


def cpu_mixed_baseline(cams, picks, seconds: float):
    """The reference CPU backend on one frame of each camera shape in `picks`,
    round robin over all host threads, for about `seconds`."""
    make, kind = cpu_pipeline_factory()
    raws = []
    for i in picks:
        c = cams[i]
        data, pitch = device_frame(c, 99)
        raws.append((c, abi.RawFrame(data.cpu().numpy(), c.width, c.height, pitch, c.fmt, c.bits, c.pattern)))
    threads = cpu_threads()
    px = 0
    t0 = time.perf_counter()
    stop = t0 + seconds

    def work(i):
        nonlocal px
        c, raw = raws[i % len(raws)]
        p = make(c.params)
        while time.perf_counter() < stop:
            p.process(raw, abi.RGB8, True)
            px += c.pixels

    ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for th in ts:
        th.start()
    for th in ts:
        th.join()
    secs = time.perf_counter() - t0
    return {"value": px / secs / 1e9, "unit": "Gpix/s", "cores": threads, "kind": kind,
            "sample": f"one frame of each of the {len(picks)} shapes, round robin over {threads} threads "
                      f"for {secs:.1f} s"}


def serving_setup(rank: int, barrier):
    """c4's 64 streams (three device-rendered fresh-seed frames each, held in
    host memory) and a runner: serve(per_frame, on_device, closed, seconds,
    clocks, copy_back) runs a server for one second of warm-up arrivals, then
    `seconds` of seeded Poisson arrivals at the nominal rates (or a closed
    loop at saturation), drains it and returns its statistics; brief(st)
    keeps the reported fields."""
    import torch

    import isp_b200

    cams, fps = scene.serving_streams()
    n_sources = 3
    sources = []
    for i, c in enumerate(cams):
        ring = []
        for k in range(n_sources):
            data, row = device_frame(c, 100_000 * (rank + 1) + 10 * i + k)
            ring.append(abi.RawFrame(data.cpu().numpy(), c.width, c.height, row, c.fmt, c.bits, c.pattern))
            del data
        sources.append(ring)
    torch.cuda.synchronize()
    budget = 8 << 30

    def make_server(per_frame: bool, on_device: bool, copy_back: bool):
        sv = isp_b200.Server(max_batch=64, max_inflight=2, queue_depth=4, slots_per_stream=2, memory_budget=budget,
                             per_frame=per_frame)
        for c, ring in zip(cams, sources):
            sid = sv.add_stream(c.params, c.width, c.height, c.fmt, c.bits, c.pattern, abi.RGB8, True, True,
                                copy_back=copy_back)
            for r in ring:
                sv.add_source(sid, r, on_device)
        sv.start()
        return sv

    def serve(per_frame: bool, on_device: bool, closed: bool, seconds: float, clocks=None, copy_back=False):
        sv = make_server(per_frame, on_device, copy_back)
        if closed:
            sv.run_closed(1.0)
        else:
            sv.run_poisson(fps, 1.0, seed=1)
        sv.drain(120.0)
        sv.reset_stats()
        barrier()
        if clocks is not None:
            clocks.start()
        if closed:
            sv.run_closed(seconds)
        else:
            sv.run_poisson(fps, seconds, seed=7 + rank)
        sv.drain(120.0)
        clock_info = clocks.stop() if clocks is not None else None
        st = sv.stats()
        sv.close()
        barrier()
        if st["error"]:
            raise RuntimeError("serving run reported a GPU-side error")
        st["clocks"] = clock_info
        return st

    def brief(st):
        return {k: st[k] for k in ("gpix_per_s", "p50_ms", "p99_ms", "p999_ms", "max_ms", "p50_wait_ms",
                                   "p99_wait_ms", "completed", "refused", "batches", "mean_batch_frames")}

    return cams, fps, budget, serve, brief


def run_serving(args):
    """Serving: 64 camera streams (four shapes, nominal 120/60/30/15 fps) with
    seeded Poisson arrivals through the continuous-batching server, against
    the same server launching each frame alone (the plain per-frame path).

    Latency percentiles come from the nominal-rate runs: a frame's latency is
    its arrival (host memory, copied to the device from pinned memory) to
    the completion of its image, histogram and statistics in device memory,
    seen by the server polling its batch's event. Throughput comes from
    closed-loop runs at saturation (every stream's queue kept full):
    completed pixels over first arrival to last completion. `value` is the
    saturation throughput with frames arriving in device memory (as from a
    capture device writing to HBM); `e2e` is the same with frames arriving in
    host memory (copied to the device per frame) and every frame's image,
    histogram and statistics copied back."""
    import torch

    import isp_b200

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    cams, fps, budget, serve, brief = serving_setup(rank, barrier)

    nominal_host = serve(False, False, False, args.seconds, Clocks(local))
    nominal_device = serve(False, True, False, args.aux_seconds)
    nominal_plain = serve(True, False, False, args.aux_seconds)
    sat_device = serve(False, True, True, args.aux_seconds, Clocks(local))
    sat_host = serve(False, False, True, args.aux_seconds, copy_back=True)
    sat_plain_device = serve(True, True, True, args.aux_seconds)
    sat_plain_host = serve(True, False, True, args.aux_seconds, copy_back=True)

    # Whole-job throughput: every rank's pixels over the slowest rank's span.
    def job(st):
        span = st["completed_pixels"] / (st["gpix_per_s"] * 1e9) if st["gpix_per_s"] > 0 else float("inf")
        return whole_job_rate(st["completed_pixels"], span, world, dist) / 1e9, span

    value, span = job(sat_device)
    e2e_value, _ = job(sat_host)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_mixed_baseline(cams, (0, 16, 40, 56), args.cpu_seconds)
    if rank == 0:
        peak, peak_kind = measured_peak()
        compulsory_per_px = sum(abi.raw_row_bytes(c.fmt, c.width) * c.height + c.pixels * 3
                                for c in cams) / sum(c.pixels for c in cams)
        achieved = value * compulsory_per_px  # Gpix/s x bytes/px = GB/s
        offered = sum(c.pixels * f for c, f in zip(cams, fps)) / 1e9
        h2d = sum(abi.raw_row_bytes(c.fmt, c.width) * c.height * f for c, f in zip(cams, fps)) / sum(fps)
        d2h = sum((c.pixels * 3 + 4096 + 48) * f for c, f in zip(cams, fps)) / sum(fps)
        line = {
            "metric": "ISP serving Gpix/s at saturation, 64 mixed streams (bit-exact); p50/p99/p99.9 at nominal rate",
            "value": value, "unit": "Gpix/s", "n_gpus": world, "steps": sat_device["completed"],
            "warmup": "1 s of arrivals per run", "ms_per_step": span * 1e3 / max(1, sat_device["completed"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene, 3 fresh-seed frames per stream in turn)",
            "config": {
                "workload": "c4_serving_64_streams",
                "streams": "16x640x480 RAW8 RGGB @120, 24x1920x1080 RAW12(u16) GBRG @60, "
                           "16x3840x2160 RAW10 GRBG @30, 8x4096x3072 RAW16 BGGR @15",
                "offered_gpix_s": offered, "memory_budget_bytes": budget, "max_batch": 64, "max_inflight": 2,
                "queue_depth": 4, "output": "RGB8 + histogram + statistics",
                "step": "one frame served", "l2": "frames rotate over 3 sources x 64 streams (1.4 GB raw) > 126 MB L2",
                "nominal_seconds": args.seconds,
                "nominal_host_arrivals": brief(nominal_host),
                "nominal_device_arrivals": brief(nominal_device),
                "nominal_per_frame_path_host_arrivals": brief(nominal_plain),
                "saturation_device_arrivals": brief(sat_device),
                "saturation_host_arrivals": brief(sat_host),
                "saturation_per_frame_path_device_arrivals": brief(sat_plain_device),
                "saturation_per_frame_path_host_arrivals": brief(sat_plain_host),
                "batched_over_per_frame_device": sat_device["gpix_per_s"] / max(1e-9, sat_plain_device["gpix_per_s"]),
                "batched_over_per_frame_host": sat_host["gpix_per_s"] / max(1e-9, sat_plain_host["gpix_per_s"]),
                "timing": "host steady clock: arrival stamps, and completion seen by the server's worker "
                          "polling each batch's done event",
                "latency": "arrival -> outputs complete in device memory (host arrivals include the copy in)",
            },
            "latency_ms": {"p50": nominal_host["p50_ms"], "p99": nominal_host["p99_ms"],
                           "p99.9": nominal_host["p999_ms"], "max": nominal_host["max_ms"],
                           "arrivals": "host memory, nominal rate"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "served batches (statistics + tile passes), device arrivals",
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gpix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "isp_b200_server_* with host-memory arrivals and result copies, saturation"},
            "gpu_launches": 3 * sat_device["batches"], "clocks": nominal_host["clocks"],
            "clocks_saturation": sat_device["clocks"],
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ---- The colour converter (the step after the ISP) ---------------------------

CC_METRIC = "colour conversion Gpix/s (bit-exact vs the reference converter)"


def cc_bytes(fmt: int, w: int, h: int) -> int:
    from isp_b200 import cc

    return cc.packed_size(fmt, w, h)


def cc_source_frames(torch, src: int, width: int, height: int, count: int):
    """`count` device frames of the synthetic camera's test pattern (frames
    0, 1, ...) converted into `src`, BT.709, as the reference's benchmark
    prepares its input."""
    from isp_b200 import cc

    conv = cc.Converter()
    rgb = torch.empty(cc.packed_size(cc.RGB8, width, height), dtype=torch.uint8, device="cuda")
    frames = []
    for i in range(count):
        cc.test_pattern(cc.packed_view(rgb.data_ptr(), cc.RGB8, width, height), i)
        buf = torch.empty(cc.packed_size(src, width, height), dtype=torch.uint8, device="cuda")
        if src == cc.RGB8:
            buf.copy_(rgb)
        else:
            conv.convert(cc.packed_view(rgb.data_ptr(), cc.RGB8, width, height),
                         cc.packed_view(buf.data_ptr(), src, width, height), cc.params(cc.BT709, mode=cc.NEAREST))
        frames.append(buf)
    torch.cuda.synchronize()
    return frames


def cc_time(torch, launch, nset: int, calls: int, rounds: int, warmup: int, stream) -> float:
    """Best over `rounds` of the mean ms per call of `calls` calls in a row,
    rotating over `nset` buffer sets, CUDA events on `stream`."""
    for i in range(warmup):
        launch(i % nset)
    best = None
    for _ in range(rounds):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i in range(calls):
            launch(i % nset)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / calls
        best = ms if best is None else min(best, ms)
    return best


def cc_graph_time(torch, launch, nset: int, calls: int) -> float:
    """Mean ms per call of `calls` calls (rotating over `nset` buffer sets)
    captured in one CUDA graph; best of three replays after a warm one."""
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        for j in range(3):
            launch(j % nset, side.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        for j in range(calls):
            launch(j % nset, side.cuda_stream)
    graph.replay()
    torch.cuda.synchronize()
    best = None
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(side)
        with torch.cuda.stream(side):
            graph.replay()
        b.record(side)
        b.synchronize()
        ms = a.elapsed_time(b) / calls
        best = ms if best is None else min(best, ms)
    del graph
    return best


def run_convert(args):
    """The colour converter: the headline case (a 3840x2160 RGB8 frame, the
    ISP's output, into NV12) timed as the contract asks, then every case of
    the reference's benchmark at 1080p and 4K timed as that benchmark does
    (best of three rounds of calls after a warm-up), beside the reference's
    own CUDA kernel built for sm_100a where oracle/_ref has it."""
    import torch

    from isp_b200 import cc
    from isp_b200.cc_workloads import BENCH_CASES, HEADLINE, SIZES

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    conv = cc.Converter()
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    src_f, dst_f, width, height = HEADLINE
    p = cc.params(cc.BT709, mode=cc.NEAREST)
    set_bytes = cc_bytes(src_f, width, height) + cc_bytes(dst_f, width, height)
    nset = max(2, math.ceil(2 * L2_BYTES / set_bytes))
    srcs = cc_source_frames(torch, src_f, width, height, nset)
    dsts = [torch.empty(cc_bytes(dst_f, width, height), dtype=torch.uint8, device="cuda") for _ in range(nset)]
    views = [(cc.packed_view(s.data_ptr(), src_f, width, height), cc.packed_view(d.data_ptr(), dst_f, width, height))
             for s, d in zip(srcs, dsts)]

    def step(i):
        sv, dv = views[i % nset]
        conv.convert(sv, dv, p, sptr)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        clocks = Clocks(local)
        clocks.start()
        time.sleep(0.3)
        barrier()
        start.record(stream)
        for i in range(args.steps):
            step(i)
        end.record(stream)
        barrier()
        clock_info = clocks.stop()
    elapsed_ms = start.elapsed_time(end)
    elapsed_max = max_over_ranks(elapsed_ms, dist)
    pixels = width * height
    value = whole_job_rate(args.steps * pixels, elapsed_ms / 1e3, world, dist) / 1e9
    kernel_ms = elapsed_ms / args.steps  # one launch per step

    # Bit-exact check of one headline output against the C oracle.
    verified = None
    if rank == 0:
        import oracle.cc as occ

        step(0)
        torch.cuda.synchronize()
        got = dsts[0].cpu().numpy()
        want = occ.convert(srcs[0].cpu().numpy(), src_f, width, height, dst_f, width, height, p, threads=16)
        verified = bool(np.array_equal(got, want))

    # End to end: pinned host frame in, converted frame out, every step.
    host_in = srcs[0].cpu().pin_memory()
    host_out = torch.empty(cc_bytes(dst_f, width, height), dtype=torch.uint8).pin_memory()
    dev_in, dev_out = srcs[0], dsts[0]
    sv, dv = views[0]
    e2e_steps = max(3, min(args.steps, 200))

    def e2e_step():
        dev_in.copy_(host_in, non_blocking=True)
        conv.convert(sv, dv, p, sptr)
        host_out.copy_(dev_out, non_blocking=True)

    with torch.cuda.stream(stream):
        for _ in range(3):
            e2e_step()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        b.record(stream)
        b.synchronize()
    e2e_sync_value = whole_job_rate(e2e_steps * pixels, a.elapsed_time(b) / 1e3, world, dist) / 1e9

    # Streamed, as a camera loop uses the asynchronous call: each frame copied
    # in from pinned host memory (upload stream), converted (compute stream)
    # and copied back (download stream), three frames in flight, so that one
    # frame's upload overlaps another's download on the full-duplex link.
    # Timed from the first upload to the last download.
    nslot = 3
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    s_in = [torch.empty_like(dev_in) for _ in range(nslot)]
    s_out = [torch.empty_like(dev_out) for _ in range(nslot)]
    h_out = [torch.empty_like(host_out).pin_memory() for _ in range(nslot)]
    s_views = [(cc.packed_view(s_in[k].data_ptr(), src_f, width, height),
                cc.packed_view(s_out[k].data_ptr(), dst_f, width, height)) for k in range(nslot)]
    ev_in = [torch.cuda.Event() for _ in range(nslot)]
    ev_done = [torch.cuda.Event() for _ in range(nslot)]
    ev_out = [torch.cuda.Event() for _ in range(nslot)]

    def streamed(i):
        k = i % nslot
        if i >= nslot:
            up.wait_event(ev_out[k])  # the slot's previous frame is back on the host
        with torch.cuda.stream(up):
            s_in[k].copy_(host_in, non_blocking=True)
        ev_in[k].record(up)
        stream.wait_event(ev_in[k])
        conv.convert(s_views[k][0], s_views[k][1], p, sptr)
        ev_done[k].record(stream)
        down.wait_event(ev_done[k])
        with torch.cuda.stream(down):
            h_out[k].copy_(s_out[k], non_blocking=True)
        ev_out[k].record(down)

    for i in range(nslot):
        streamed(i)
    torch.cuda.synchronize()
    barrier()
    ta, tb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ta.record(up)
    for i in range(e2e_steps):
        streamed(i)
    tb.record(down)
    tb.synchronize()
    e2e_value = whole_job_rate(e2e_steps * pixels, ta.elapsed_time(tb) / 1e3, world, dist) / 1e9

    # Every case of the reference's benchmark, ours beside the reference kernel's.
    cases = []
    have_ref = False
    if rank == 0 and not args.no_cases:
        import oracle.cc as occ

        have_ref = occ.have_ref_cuda()
        calls = max(20, min(200, args.steps))
        for w, h in SIZES:
            for src, dst, ow, oh, mode, box, label in BENCH_CASES:
                dw, dh = ow or w, oh or h
                cp = cc.params(cc.BT709, mode=mode, letterbox=box)
                per = cc_bytes(src, w, h) + cc_bytes(dst, dw, dh)
                k = max(2, math.ceil(2 * L2_BYTES / per))
                ins = cc_source_frames(torch, src, w, h, 1) * k
                outs = [torch.empty(cc_bytes(dst, dw, dh), dtype=torch.uint8, device="cuda") for _ in range(k)]
                ins = [i.clone() for i in ins]
                vv = [(cc.packed_view(i.data_ptr(), src, w, h), cc.packed_view(o.data_ptr(), dst, dw, dh))
                      for i, o in zip(ins, outs)]
                with torch.cuda.stream(stream):
                    ours = cc_time(torch, lambda j: conv.convert(vv[j][0], vv[j][1], cp, sptr), k, calls, 3, 50, stream)
                    ref = None
                    if have_ref:
                        ref = cc_time(torch, lambda j: occ.ref_cuda_convert(vv[j][0], vv[j][1], cp, sptr), k, calls, 3,
                                      50, stream)
                # The same calls captured once in a CUDA graph and replayed: the
                # kernels without the host launch path (both implementations).
                ours_g = cc_graph_time(torch, lambda j, sp: conv.convert(vv[j][0], vv[j][1], cp, sp), k, calls)
                ref_g = None
                if have_ref:
                    ref_g = cc_graph_time(torch, lambda j, sp: occ.ref_cuda_convert(vv[j][0], vv[j][1], cp, sp), k,
                                          calls)
                cases.append({"input": f"{cc.format_name(src)} {w}x{h}", "output": f"{cc.format_name(dst)} {dw}x{dh}",
                              "operation": label, "ms": round(ours, 5),
                              "reference_kernel_ms": None if ref is None else round(ref, 5),
                              "speedup": None if ref is None else round(ref / ours, 3),
                              "gbs": round(per / (ours / 1e3) / 1e9, 1),
                              "graph_ms": round(ours_g, 5),
                              "reference_kernel_graph_ms": None if ref_g is None else round(ref_g, 5),
                              "graph_speedup": None if ref_g is None else round(ref_g / ours_g, 3)})
                del ins, outs, vv

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cc_cpu_baseline(args.cpu_seconds, cpu_threads())

    if dist is not None:
        dist.barrier()
    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = set_bytes / (kernel_ms / 1e3) / 1e9
        line = {
            "metric": CC_METRIC, "value": value, "unit": "Gpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (the reference benchmark's "
            "test pattern)",
            "config": {"workload": "convert_rgb8_to_nv12_3840x2160", "source": "rgb8 3840x2160",
                       "destination": "nv12 3840x2160", "matrix": "bt709", "range": "limited",
                       "compulsory_bytes_per_frame": set_bytes,
                       "l2": f"{nset} rotating buffer sets, {nset * set_bytes / 1e6:.0f} MB > 126 MB L2",
                       "verified_bit_exact": verified},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profiled_traffic("cc_direct_kernel", "convert"), "kernel": "cc_direct_kernel",
                         "kernel_ms": kernel_ms, "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gpix/s", "h2d_bytes_per_step": cc_bytes(src_f, width, height),
                    "d2h_bytes_per_step": cc_bytes(dst_f, width, height), "steps": e2e_steps,
                    "api": "cc_b200_convert with pinned-host uploads and downloads on their own streams, "
                           "three frames in flight",
                    "synchronous_value": e2e_sync_value,
                    "synchronous_api": "upload, cc_b200_convert, download in turn on one stream"},
            "gpu_launches": args.steps,
            "clocks": clock_info,
            "cases": cases,
            "reference_kernel": "oracle/_ref/libcc_ref_cuda.so (the reference's kernels.cu, sm_100a, --fmad=false)"
            if have_ref else None,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cc_cpu_baseline(seconds: float, threads: int):
    """The reference's reference_convert (oracle/_ref, else the C oracle) on
    the host cores: `threads` independent 4K RGB8 -> NV12 conversions at a
    time for about `seconds`."""
    import oracle.cc as occ
    from isp_b200 import cc
    from isp_b200.cc_workloads import HEADLINE

    src_f, dst_f, w, h = HEADLINE
    img = occ.test_pattern(w, h, 0)
    kind = "reference" if occ.have_ref() else "port"
    fn = occ.ref_convert if kind == "reference" else occ.convert
    p = cc.params(cc.BT709, mode=cc.NEAREST)
    fn(img, src_f, w, h, dst_f, w, h, p)
    counts = [0] * threads
    stop = time.perf_counter() + seconds

    def work(i):
        while time.perf_counter() < stop or counts[i] == 0:
            fn(img, src_f, w, h, dst_f, w, h, p)
            counts[i] += 1

    t0 = time.perf_counter()
    ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    secs = time.perf_counter() - t0
    frames = sum(counts)
    return {"value": frames * w * h / secs / 1e9, "unit": "Gpix/s", "cores": threads, "kind": kind,
            "sample": f"{frames} frames rgb8->nv12 {w}x{h} over {secs:.1f} s on {threads} threads"}


def run_convert_reference(args):
    """--impl reference --workload convert: the reference's reference_convert
    on the host cores, the headline case, each step every thread converting
    one frame."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle.cc as occ
    from isp_b200 import cc
    from isp_b200.cc_workloads import HEADLINE

    src_f, dst_f, w, h = HEADLINE
    threads = cpu_threads()
    img = occ.test_pattern(w, h, 0)
    kind = "reference" if occ.have_ref() else "port"
    fn = occ.ref_convert if kind == "reference" else occ.convert
    p = cc.params(cc.BT709, mode=cc.NEAREST)

    def step():
        t0 = time.perf_counter()
        ts = [threading.Thread(target=fn, args=(img, src_f, w, h, dst_f, w, h, p)) for _ in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    times = []
    for i in range(min(args.warmup, 3) + min(args.steps, 20)):
        t = step()
        if i >= min(args.warmup, 3):
            times.append(t)
    total = sum(times)
    value = threads * w * h * len(times) / total / 1e9
    line = {
        "metric": CC_METRIC, "value": value, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": len(times),
        "warmup": min(args.warmup, 3), "ms_per_step": total / len(times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (the reference benchmark's test pattern)",
        "config": {"workload": "convert_rgb8_to_nv12_3840x2160"}, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Gpix/s", "cores": threads, "kind": kind,
                         "sample": f"{threads} threads x one {w}x{h} frame per step"},
        "e2e": {"value": value, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- The demo's side-by-side view -------------------------------------------

VIEW_METRIC = "side-by-side view Gpix/s (bit-exact vs the C restatement)"


def run_view(args):
    """isp_b200_view_compose on a 3840x2160 RAW10 frame and its RGB8 image
    into the 7680x2160 RGB8 view: device-resident throughput over rotating
    buffer sets larger than L2, the kernel's roofline, and the C restatement
    (oracle_view_compose) on the host cores as the CPU baseline (the demo's
    own kernel needs the Holoscan SDK)."""
    import torch

    import isp_b200
    import oracle

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    w, h, black = 3840, 2160, 64.0
    rng = np.random.default_rng(5 + rank)
    pitch = abi.raw_row_bytes(abi.RAW10, w)
    raw = abi.RawFrame(rng.integers(0, 256, pitch * h, dtype=np.uint8), w, h, pitch, abi.RAW10, 10, abi.GRBG)
    rgb = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    per = pitch * h + 3 * w * h + 6 * w * h
    nset = max(2, math.ceil(2 * L2_BYTES / per))
    d_raw = [torch.from_numpy(raw.data).cuda() for _ in range(nset)]
    d_rgb = [torch.from_numpy(rgb.reshape(-1)).cuda() for _ in range(nset)]
    d_out = [torch.empty(6 * w * h, dtype=torch.uint8, device="cuda") for _ in range(nset)]
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    def step(i):
        k = i % nset
        isp_b200.view_compose(raw.view(d_raw[k].data_ptr()), black, d_rgb[k].data_ptr(), 3 * w, d_out[k].data_ptr(),
                              6 * w, sptr)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
        torch.cuda.synchronize()
        clocks = Clocks(local)
        clocks.start()
        time.sleep(0.3)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i in range(args.steps):
            step(i)
        b.record(stream)
        b.synchronize()
        clock_info = clocks.stop()
    ms = a.elapsed_time(b) / args.steps
    value = whole_job_rate(args.steps * w * h, ms * args.steps / 1e3, world, None) / 1e9
    got = d_out[0].cpu().numpy().reshape(h, 2 * w, 3)
    verified = bool(np.array_equal(got, oracle.view_compose(raw, black, rgb)))

    # End to end: the raw frame and the RGB8 image from pinned host memory, the view back, every step.
    h_raw = torch.from_numpy(raw.data).pin_memory()
    h_rgb = torch.from_numpy(rgb.reshape(-1)).pin_memory()
    h_out = torch.empty(6 * w * h, dtype=torch.uint8).pin_memory()
    e2e_steps = max(3, min(args.steps, 100))
    with torch.cuda.stream(stream):
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        for _ in range(e2e_steps):
            d_raw[0].copy_(h_raw, non_blocking=True)
            d_rgb[0].copy_(h_rgb, non_blocking=True)
            step(0)
            h_out.copy_(d_out[0], non_blocking=True)
        eb.record(stream)
        eb.synchronize()
    e2e_value = e2e_steps * w * h / (ea.elapsed_time(eb) / 1e3) / 1e9

    cpu = None
    if not args.no_cpu_baseline:
        threads = cpu_threads()
        rows = 64
        band = abi.RawFrame(raw.data[: rows * pitch], w, rows, pitch, abi.RAW10, 10, abi.GRBG)
        counts = [0] * threads
        stop = time.perf_counter() + args.cpu_seconds

        def work(i):
            while time.perf_counter() < stop or counts[i] == 0:
                oracle.view_compose(band, black, rgb[:rows])
                counts[i] += 1

        t0 = time.perf_counter()
        ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        secs = time.perf_counter() - t0
        cpu = {"value": sum(counts) * w * rows / secs / 1e9, "unit": "Gpix/s", "cores": threads, "kind": "port",
               "sample": f"{sum(counts)} bands of {w}x{rows} over {secs:.1f} s on {threads} threads"}

    peak, peak_kind = measured_peak()
    achieved = per / (ms / 1e3) / 1e9
    line = {
        "metric": VIEW_METRIC, "value": value, "unit": "Gpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (random RAW10 frame and RGB8 image)",
        "config": {"workload": "view_3840x2160_raw10", "view": "7680x2160 RGB8", "black_level": black,
                   "compulsory_bytes_per_frame": per,
                   "l2": f"{nset} rotating buffer sets, {nset * per / 1e6:.0f} MB > 126 MB L2",
                   "verified_bit_exact": verified},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "isp_view_kernel", "kernel_ms": ms, "peak_kind": peak_kind},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "Gpix/s", "h2d_bytes_per_step": pitch * h + 3 * w * h,
                "d2h_bytes_per_step": 6 * w * h, "steps": e2e_steps,
                "api": "isp_b200_view_compose between pinned-host copies, one stream"},
        "gpu_launches": args.steps,
        "clocks": clock_info,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_view_reference(args):
    """--impl reference --workload view: the demo's view kernel needs the
    Holoscan SDK, so the reference arm times its C restatement
    (oracle_view_compose) on the host cores, bands of the same frame."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle

    w, rows, black = 3840, 64, 64.0
    rng = np.random.default_rng(5)
    pitch = abi.raw_row_bytes(abi.RAW10, w)
    band = abi.RawFrame(rng.integers(0, 256, pitch * rows, dtype=np.uint8), w, rows, pitch, abi.RAW10, 10, abi.GRBG)
    rgb = rng.integers(0, 256, (rows, w, 3), dtype=np.uint8)
    threads = cpu_threads()

    def step():
        t0 = time.perf_counter()
        ts = [threading.Thread(target=oracle.view_compose, args=(band, black, rgb)) for _ in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    times = []
    for i in range(min(args.warmup, 3) + min(args.steps, 50)):
        t = step()
        if i >= min(args.warmup, 3):
            times.append(t)
    total = sum(times)
    value = threads * w * rows * len(times) / total / 1e9
    line = {
        "metric": VIEW_METRIC, "value": value, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": len(times),
        "warmup": min(args.warmup, 3), "ms_per_step": total / len(times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (random RAW10 frame and RGB8 image)",
        "config": {"workload": "view_3840x2160_raw10"}, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Gpix/s", "cores": threads, "kind": "port",
                         "sample": f"{threads} threads x one {w}x{rows} band per step"},
        "e2e": {"value": value, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference" and args.workload == "view":
        run_view_reference(args)
    elif args.impl == "reference" and args.workload == "convert":
        run_convert_reference(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "convert":
        run_convert(args)
    elif args.workload == "view":
        run_view(args)
    elif args.workload == "c3":
        run_batch(args)
    elif args.workload == "c4":
        run_serving(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
