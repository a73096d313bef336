#!/usr/bin/env python
"""Benchmark of the sliding-window outlier detector on one or more B200s.

Workload (N=1): the stock-like 1-d stream standing in for RTOD's STK run
(script/run.py:25): 1,048,572 float32 values (random walk, N(0, 0.1) steps,
0.5% U(-5, 5) jumps, seed 1), W=100,000, S=5,000, R=0.45, K=50,
FP32 predicate, 189 slides. One step = one pass over the whole stream, as in
RTOD's timed pass (src/ods/optixScan.cpp:1159-1168): fill with the first W
points, then detect every slide.

  value   stream points ingested per second (S * slides / step time), the
          stream resident in HBM, outputs left in HBM; device time from CUDA
          events on the library's stream, summed over the timed steps, max
          over ranks; L2 flushed (256 MiB write) before every step.
  e2e     the same through the public API with host buffers: pinned host
          input copied in and the outlier IDs copied out inside every step;
          host wall clock around each call (the call synchronises).

Multi-GPU: replicas only (independent streams, no collective); every rank
runs the same workload and value counts the points of all ranks.

`--impl reference` times the CPU restatement of RTOD's detection path
(oracle/, grid filter + exact count, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "µs/slide & points/s: learned-routed vs plain kernel, 1 B200, bit-exact outliers"
UNIT = "points/s"
FLUSH_BYTES = 256 << 20
KERNEL_ORDER = ["k_ingest", "k_hist", "k_scan", "k_scatter", "k_count", "k_compact"]


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-stream multi-stream measurement")
    ap.add_argument("--mode", choices=["bench", "ncu", "ncu-stream", "ncu-stream-grid", "ncu-batched",
                                       "replica-check"],
                    default="bench",
                    help="ncu: passes of the headline workload inside a cudaProfilerStart/Stop range; "
                         "ncu-stream(-grid): 30 push/detect slides of it (window or grid engine) inside one; "
                         "ncu-batched: 2 multi-stream steps of the 8-d streams of the 64-stream workload "
                         "inside one; "
                         "replica-check: the multi-rank plumbing on host ranks (gloo), no GPU")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Ranks:
    """Replica plumbing: one process per GPU, each detecting its own copy of
    the workload; no collective on the data path. Only barriers and the
    maximum of the device-timed durations cross ranks (backend "nccl" on
    GPUs, "gloo" on the host)."""

    def __init__(self, world: int, backend: str, device: str):
        import datetime
        import torch.distributed as dist
        self.world, self.device, self.dist = world, device, dist
        if world > 1:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))

    def barrier(self):
        import torch
        if self.device.startswith("cuda"):
            torch.cuda.synchronize()
        if self.world > 1:
            self.dist.barrier()

    def reduce(self, x: float, op: str = "max") -> float:
        import torch
        if self.world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.MIN)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def workload():
    from rtod_b200 import datagen
    return datagen.stock_like()


def workload_config(w, extra=None):
    cfg = {"workload": w.name, "stream_points": w.n, "dim": w.dim, "window": w.window,
           "slide": w.slide, "R": w.R, "K": w.K, "slides_per_step": w.slides,
           "predicate": "fp32 d2 <= R2", "l2": "flushed before every step (256 MiB write)",
           "parallelism": "replicas"}
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 50 ms while the
    timed region runs; entering waits (up to 5 s) for the first sample so
    that short regions are covered too."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = threading.Event()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)
            self.first.set()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        self.first.wait(5.0)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self.reader.join(timeout=5)
        self.out = "".join(self.lines)

    def summary(self):
        rows = [r for r in csv.reader(io.StringIO(self.out or "")) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def physical_gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        parts = [p.strip() for p in vis.split(",") if p.strip()]
        if local_rank < len(parts) and parts[local_rank].isdigit():
            return int(parts[local_rank])
    return local_rank


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary
    (profiles/ncu_traffic.txt lines: `<kernel> <workload> <bytes per launch>`)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and parts[0] == kernel and not line.startswith("#"):
                return float(parts[2])
    except OSError:
        pass
    return None


def pass_roofline(w, n_out_per_slide: float, us_per_slide: float, peak: float) -> dict:
    """Bytes per slide that a detector reading every window point once per
    slide moves (new slide in, ring write, one read of the window, IDs out),
    against the measured device time per slide of the whole pass."""
    d = w.dim
    per_slide = 4 * d * w.slide + 4 * d * w.slide + 4 * d * w.window + 4 * n_out_per_slide
    achieved = per_slide / (us_per_slide * 1e-6) / 1e9
    return {"algorithmic_bytes_per_slide": per_slide, "us_per_slide": us_per_slide,
            "achieved": achieved, "unit": "GB/s", "frac": achieved / peak}


def used_bins(w, cells_per_r: int, batch: int) -> int:
    """Bins of the 65536-bin table holding points of the first span of
    `batch` windows (1-d cells of R(1+2^-12)/n, bin = cell mod 65536)."""
    span = w.points[w.slide:w.slide + w.window + (batch - 1) * w.slide, 0].astype(np.float64)
    cell = w.R * (1 + 2.0 ** -12) / cells_per_r
    return int(np.unique(np.floor(span / cell).astype(np.int64) & 65535).size)


def algorithmic_bytes(kernel: str, w, n_out_per_slide: float, undet_per_slide: float, batch: int,
                      used_bins: int = 0) -> float:
    """Minimum DRAM bytes of each pipeline stage per slide (per window); the
    span engine's stages move their per-batch bytes once per `batch` windows."""
    W, S, d = w.window, w.slide, w.dim
    span_pts = (W // S + batch - 1) * S  # points of one span of `batch` windows
    return {
        "k_ingest": 4 * d * S + 4 * d * S + 8 * S,           # read slide, write ring + keys
        "k_hist": 8 * W,                                      # read every key
        "k_scan": 4 * 65536 * 3,                              # read counts, write starts+cursors
        "k_scatter": 8 * W + 4 * d * W + (4 + 8 + 4 * d) * W,  # read keys+ring, write SoA
        "k_count": (8 + 4 + 4 * d) * W,                       # read the cell-ordered SoA once
        "k_compact": W / 8 + 8 * n_out_per_slide,             # read the outlier bits, write IDs
        "k_keys": 4 * d * S + 8 * S,                          # per slide: read points, write keys
        "k_train": 2048 * 16 + 3 * 1316 * 4 * 2,              # samples + params/moments (per batch)
        # span engine: read the span's points, write their keys, once per batch
        "k_span_hist": (4 * d + 8) * span_pts / batch,
        # read counts, write starts; per bin in use, its per-block counts and prefixes
        "k_span_scan+k_span_prefix": (4 * 65536 * 2 + 8 * used_bins * (W // S + batch)) / batch,
        # read keys + points, write bin-ordered offsets + coordinates, once per batch
        "k_span_scatter": ((8 + 4 * d) + (4 + 4 * d)) * span_pts / batch,
        # per (window, bin in use): the bin's two prefix entries
        "k_span_classify": 8 * used_bins,
        # per counted point: its offset and coordinates (candidates are read
        # per group of one bin and shared by its points: not counted)
        "k_span_count": undet_per_slide * (4 + 4 * d),
        # per slide: its bitset row, its outlier IDs
        "k_span_compact": W / 8 + 8 * n_out_per_slide,
    }[kernel]


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch
    from rtod_b200 import Detector

    torch.cuda.set_device(local)
    ranks = Ranks(world, "nccl", f"cuda:{local}")
    w = workload()
    slides = w.slides
    cap = slides * w.window // 4
    pts_dev = torch.from_numpy(w.points).to(f"cuda:{local}")
    out_dev = torch.empty(cap, dtype=torch.int64, device=f"cuda:{local}")
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")

    barrier = ranks.barrier
    max_over_ranks = ranks.reduce

    def measure(kw, steps, full):
        """Device-timed passes of one engine configuration; with full=True also
        the clocks, the end-to-end passes and the per-kernel profile."""
        det = Detector(w.window, w.slide, w.R, w.K, dim=w.dim, device=local, **kw)
        ref = None
        for _ in range(max(3, args.warmup)):
            det.reset()
            r = det.run(pts_dev, out_ids=out_dev, ids_cap=cap, times=True)
            ref = r.offsets.copy()
        ids_ref = out_dev[:int(ref[-1])].cpu().numpy()
        stats0 = det.stats
        barrier()
        dev_ms = 0.0
        with ClockSampler(physical_gpu_index(local)) as clk:
            for _ in range(steps):
                flush.zero_()
                torch.cuda.synchronize()
                det.reset()
                r = det.run(pts_dev, out_ids=out_dev, ids_cap=cap, times=True)
                dev_ms += r.times["total"] * r.slides
        barrier()
        stats1 = det.stats
        assert np.array_equal(r.offsets, ref)
        out = dict(dev_ms=max_over_ranks(dev_ms), steps=steps, offsets=ref, ids=ids_ref,
                   launches=stats1["launches"] - stats0["launches"],
                   undet=r.times["undetermined_per_slide"], n_outliers=int(ref[-1]))
        if full:
            out["clocks"] = clk.summary()
            # end to end through the public API with pinned host buffers
            pts_pin = torch.from_numpy(w.points).pin_memory()
            ids_pin = torch.empty(cap, dtype=torch.int64).pin_memory()
            pts_np, ids_np = pts_pin.numpy(), ids_pin.numpy()
            for _ in range(2):
                det.reset()
                det.run(pts_np, out_ids=ids_np, ids_cap=cap)
            barrier()
            e2e_s = 0.0
            e2e_steps = max(3, min(steps, 50))
            for _ in range(e2e_steps):
                flush.zero_()
                torch.cuda.synchronize()
                det.reset()
                t0 = time.perf_counter()
                r2 = det.run(pts_np, out_ids=ids_np, ids_cap=cap)
                e2e_s += time.perf_counter() - t0
            barrier()
            assert np.array_equal(r2.offsets, ref) and np.array_equal(r2.ids, ids_ref)
            out.update(e2e_s=max_over_ranks(e2e_s), e2e_steps=e2e_steps, h2d=w.n * w.dim * 4,
                       d2h=(slides + 1) * 8 + out["n_outliers"] * 8 + slides * 8)
            # per-kernel device time of one pass (diagnostic, individual launches)
            det.reset()
            out["prof"] = det.profile(pts_dev)
            out["tuning"] = det.tuning
            if kw.get("router"):
                info = det.router_info()
                out["router"] = {k: info[k] for k in ("steps", "last_loss", "routed_early",
                                                      "routed_sweep", "misrouted")}
        det.close()
        return out

    results = {
        # headline: the autotuner picks the engine (span / window with the learned
        # router), cell width, block shape and windows per launch
        "tuned": measure(dict(router=True, tuner=True), args.steps, True),
        # span engine, default settings: one counting sort per batch of windows
        "span": measure(dict(engine="span"), args.steps, False),
        # window engine with the learned router on
        "window_routed": measure(dict(engine="window", router=True), args.steps, False),
        # window engine, router off, 32 windows per launch
        "window_batched": measure(dict(engine="window"), args.steps, False),
        # window engine, one window per launch (graph replay per slide)
        "window_single": measure(dict(engine="window", batch=1), args.steps, False),
    }
    base = results["tuned"]
    for name, r in results.items():
        assert np.array_equal(r["offsets"], base["offsets"]), name
        assert np.array_equal(r["ids"], base["ids"]), name
    base["streaming"] = measure_streaming(w, local, base)
    base["batched"] = None if args.no_batched else measure_batched(local)
    base["router_ab"] = measure_router_ab(local)
    ranks.close()
    if rank != 0:
        return None
    return w, results


def measure_streaming(w, local, base, slides: int = 60):
    """RTOD's own per-slide loop through the public API: push S points from
    host memory, detect, read the IDs back (host wall clock per slide, after
    10 untimed slides), with the window engine (the default of push/detect)
    and with the streaming grid engine; the IDs must match the whole-stream
    run. The device time of a slide comes from a second pass
    with per-detection stage times (CUDA events around the detection's
    launches). The native command line (C++ over the C ABI, no Python in the
    loop) runs the same loop on the whole stream."""
    from rtod_b200 import Detector
    W, S = w.window, w.slide
    n = min(slides, w.slides)
    out = {"slides": n, "api": "rtod_push_slide + rtod_detect, host arrays"}
    for engine in ("grid", "window"):
        ts, dev = [], []
        with Detector(W, S, w.R, w.K, dim=w.dim, device=local, engine=engine) as det:
            for timed in (False, True):
                det.reset()
                det.push(w.points[:W])
                for j in range(n):
                    t0 = time.perf_counter()
                    det.push(w.points[W + j * S:W + (j + 1) * S])
                    got = det.detect(times=timed)
                    t1 = time.perf_counter()
                    ids = got[0] if timed else got
                    if timed:
                        dev.append(got[1]["total"] * 1e3)
                    else:
                        ts.append(t1 - t0)
                    assert np.array_equal(ids, base["ids"][base["offsets"][j]:base["offsets"][j + 1]])
            info = det.stream_engine
        out[engine] = {"us_per_slide_wall": float(np.median(ts[10:])) * 1e6,
                       "us_per_slide_device": float(np.median(dev[10:])),
                       "engine": info["engine"], "grid_builds": info["builds"]}
    out["us_per_slide_wall"] = out["window"]["us_per_slide_wall"]
    out["native"] = native_streaming(w, local, base)
    return out


def native_streaming(w, local, base):
    """The native rtod command line in its --streaming mode (RTOD's per-slide
    loop in C++ through rtod_push_slide + rtod_detect) on the same stream,
    written in RTOD's text format: median wall time per slide, its outliers
    checked against the whole-stream run."""
    import subprocess
    import tempfile
    from rtod_b200 import build
    exe = os.path.join(os.path.dirname(build.LIB), "rtod")
    if not os.path.exists(exe):
        return None
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "stream.txt")
        np.savetxt(path, w.points.reshape(len(w.points), -1).astype(np.float64), fmt="%.9g",
                   delimiter=",")
        res = {}
        for engine in ("grid", "window"):
            cmd = [exe, "-f", path, "--n", str(len(w.points)), "--window", str(w.window), "--slide", str(w.slide),
                   "--R", repr(float(w.R)), "--K", str(w.K), "--dim", str(w.dim), "--streaming", "--engine",
                   engine, "--warmup", "10", "--device", str(local), "--print-outliers"]
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                return {"error": r.stderr.strip()[-300:]}
            wall = [ln for ln in r.stdout.splitlines() if ln.startswith("[Wall]")]
            total = [ln for ln in r.stdout.splitlines() if ln.startswith("[Time] total time for a slide")]
            rows = [ln for ln in r.stdout.splitlines() if ln.startswith("slide ")]
            same = len(rows) == w.slides and all(
                np.array_equal(np.array(ln.split(":", 1)[1].split(), dtype=np.int64),
                               base["ids"][base["offsets"][j]:base["offsets"][j + 1]])
                for j, ln in enumerate(rows))
            res[engine] = {"us_per_slide_wall_median": float(wall[0].split("median:")[1].split("us")[0]),
                           "us_per_slide_device": float(total[0].split(":")[1].split("ms")[0]) * 1e3,
                           "slides": len(rows), "same_outliers": bool(same)}
    res["api"] = "rtod --streaming (C++), rtod_push_slide + rtod_detect from host arrays"
    return res


# FP32 operations of one distance test under the FP32 predicate in d
# dimensions: d subtractions, d multiplies, d-1 adds (no FMA contraction)
# and a compare.
OPS_PER_TEST = {d: 3 * d for d in range(1, 9)}


def measure_batched(local, steps: int = 20, warmup: int = 3, tune_max: int = 24):
    """The batched workload: 64 independent streams (W log-uniform in [5k,
    200k], S = W/20, d in {1, 3, 8}) through the multi-stream API, one graph
    replay per step: with the autotuner (each group's cell width, count block
    shape and count mode tried over the first steps, untimed, then fixed),
    with the learned router on as well, with the default settings, and with
    the persistent fused launch. The step time is the wall time of
    rtod_batch_step (it ends with one stream wait); e2e adds the step's 64
    host pushes. The 8-d streams also run alone, to set their group count's
    distance tests against the FP32 issue rate (compute bound: every point
    is counted against thousands of candidates)."""
    import torch
    from rtod_b200 import BatchDetector, datagen
    streams = datagen.batched_streams(slides=tune_max + warmup + steps)
    pts_per_step = sum(s.slide for s in streams)

    def run(subset, pipeline="staged", tuner=False, router=False):
        cfg = [dict(window=s.window, slide=s.slide, R=s.R, K=s.K, dim=s.dim, pipeline=pipeline) for s in subset]
        with BatchDetector(cfg, device=local, tuner=tuner, router=router) as bd:
            for i, s in enumerate(subset):
                bd.push(i, s.points[:s.window])
            t_step, t_e2e = [], []
            tests0 = 0
            j = 0

            def one(timed):
                nonlocal j
                t0 = time.perf_counter()
                for i, s in enumerate(subset):
                    bd.push(i, s.points[s.window + j * s.slide:s.window + (j + 1) * s.slide])
                t1 = time.perf_counter()
                bd.step()
                t2 = time.perf_counter()
                j += 1
                if timed:
                    t_step.append(t2 - t1)
                    t_e2e.append(t2 - t0)

            while tuner and j < tune_max and not all(g["settled"] for g in bd.tuning):
                one(False)
            tune_steps = j
            for _ in range(warmup):
                one(False)
            tests0 = bd.stats["pair_tests"]
            for _ in range(steps):
                one(True)
            st = bd.stats
            return (float(np.sum(t_step)), float(np.sum(t_e2e)), st, st["pair_tests"] - tests0,
                    {"tuning_steps": tune_steps, "groups": bd.tuning})

    torch.cuda.synchronize()
    with ClockSampler(physical_gpu_index(local)) as clk:
        t_step, t_e2e, st, _, tinfo = run(streams, tuner=True)
    t_plain, _, _, _, _ = run(streams)
    t_router, _, _, _, rinfo = run(streams, tuner=True, router=True)
    t_fused, _, _, _, _ = run(streams, "fused")
    d8 = [s for s in streams if s.dim == 8]
    t8, _, _, tests8, _ = run(d8, tuner=True)
    sm = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = clk.summary()["sm_mhz"] or 1965.0
    peak_ops = sm * 128 * mhz * 1e6  # FP32 lanes x clock: one FP32 operation per lane and cycle
    achieved_ops = tests8 * OPS_PER_TEST[8] / t8
    return {
        "workload": "64 streams, W log-uniform in [5k, 200k], S = W/20, d in {1, 3, 8}, ~2% outliers, K = 50",
        "streams": len(streams), "by_dim": {d: sum(s.dim == d for s in streams) for d in (1, 3, 8)},
        "steps": steps, "ms_per_step": t_step / steps * 1e3, "points_per_s": pts_per_step * steps / t_step,
        "window_points_per_s": sum(s.window for s in streams) * steps / t_step,
        "e2e": {"ms_per_step": t_e2e / steps * 1e3, "points_per_s": pts_per_step * steps / t_e2e,
                "h2d_bytes_per_step": sum(4 * s.dim * s.slide for s in streams)},
        "autotuner": dict(tinfo, untuned_ms_per_step=t_plain / steps * 1e3),
        "router_on": {"ms_per_step": t_router / steps * 1e3, "tuning_steps": rinfo["tuning_steps"]},
        "fused_pipeline_ms_per_step": t_fused / steps * 1e3,
        "launches_per_step": st["launches"] / max(1, st["steps"]), "groups": st["groups"],
        "clocks": clk.summary(),
        "roofline_8d": {"bound": "fp32 issue", "streams": len(d8), "ms_per_step": t8 / steps * 1e3,
                        "distance_tests_per_step": tests8 / steps, "ops_per_test": OPS_PER_TEST[8],
                        "achieved": achieved_ops / 1e12, "peak": peak_ops / 1e12, "unit": "TFLOP/s (FP32 ops)",
                        "frac": achieved_ops / peak_ops,
                        "peak_source": f"{sm} SMs x 128 FP32 lanes x {mhz:.0f} MHz (median SM clock sampled)"},
    }


def measure_router_ab(local, steps: int = 11):
    """The learned router on and off, both autotuned, on the configurations
    that name it (sensor-like 3-d: router on; Gaussian mixture K=30: router
    vs plain) and the headline stream: device time per slide (median over
    steps passes, device-resident stream and outputs), outliers identical."""
    import torch
    from rtod_b200 import Detector, datagen
    out = {}
    for w in (datagen.stock_like(), datagen.sensor_like(), datagen.gaussian_like(30)):
        pts = torch.from_numpy(w.points).to(f"cuda:{local}")
        cap = w.slides * w.window // 4 + 1024
        ids = torch.empty(cap, dtype=torch.int64, device=f"cuda:{local}")
        row, ref = {}, None
        for router in (False, True):
            with Detector(w.window, w.slide, w.R, w.K, dim=w.dim, device=local, tuner=True, router=router) as det:
                ts = []
                for _ in range(3 + steps):
                    det.reset()
                    r = det.run(pts, out_ids=ids, ids_cap=cap, times=True)
                    ts.append(r.times["total"] * 1e3)
                got = (r.offsets.copy(), ids[:int(r.offsets[-1])].cpu().numpy())
                if ref is None:
                    ref = got
                assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
                key = "router_on" if router else "router_off"
                row[key] = {"us_per_slide": float(np.median(ts[3:])), "tuning": det.tuning}
                if router:
                    info = det.router_info()
                    row[key]["router"] = {k: info[k] for k in ("steps", "routed_early", "routed_sweep", "misrouted")}
        row["speedup"] = row["router_off"]["us_per_slide"] / row["router_on"]["us_per_slide"]
        row["bit_exact"] = True
        out[w.name] = row
    return out


def cpu_baseline(w):
    """The oracle's grid engine (CPU restatement of RTOD's path) on the whole
    stream: all host threads (the reported value) and one thread."""
    from oracle import oracle
    oracle.build()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    off, ids, st = oracle.detect(w.points, w.window, w.slide, w.R, w.K, engine="grid", threads=threads)
    dt = time.perf_counter() - t0
    t0 = time.perf_counter()
    off1, ids1, _ = oracle.detect(w.points, w.window, w.slide, w.R, w.K, engine="grid", threads=1)
    dt1 = time.perf_counter() - t0
    assert np.array_equal(off, off1) and np.array_equal(ids, ids1)
    slides = len(off) - 1
    return {"value": slides * w.slide / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"whole stream once ({slides} slides), oracle grid engine, slides split over "
                      f"{threads} threads", "us_per_slide": dt / slides * 1e6,
            "single_thread": {"value": slides * w.slide / dt1, "unit": UNIT, "cores": 1,
                              "us_per_slide": dt1 / slides * 1e6}}, (off, ids)


def emit_ours(args, world, w, res):
    r = res["tuned"]
    K = args.steps
    slides = w.slides
    t_s = r["dev_ms"] / 1e3
    value = world * K * slides * w.slide / t_s
    us_slide = r["dev_ms"] * 1e3 / (K * slides)
    # roofline of the dominant kernel
    prof = r["prof"]
    dom = max(prof, key=prof.get)
    n_out = r["n_outliers"] / slides
    tun = r["tuning"]
    batch = min(tun["batch"], slides)  # windows per launch of the pipeline kernels
    ub = used_bins(w, tun["cells_per_r"], batch) if w.dim == 1 else 0
    alg = algorithmic_bytes(dom, w, n_out, r["undet"], batch, ub)
    peak, peak_kind = hbm_peak()
    # per launch: pipeline kernels run once per batch of windows, the key
    # kernel and the chunk compaction once per pass over the stream
    per_launch = slides if dom in ("k_keys", "k_span_compact") else batch
    launch_ms = prof[dom] * per_launch
    # achieved: the per-slide algorithmic bytes of the detector (4dS slide in,
    # 4dS ring write, 4dW window read, 4 n_out IDs out) times the windows one
    # launch of the dominant kernel serves, over that launch's device time
    slide_bytes = 4 * w.dim * w.slide * 2 + 4 * w.dim * w.window + 4 * n_out
    achieved = slide_bytes * per_launch / (launch_ms / 1e3) / 1e9
    traffic = ncu_traffic(dom)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": r["dev_ms"] / K, "us_per_slide": us_slide,
        "window_points_per_s": world * K * slides * w.window / t_s,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded stand-in for RTOD's STK stream)",
        "config": workload_config(w),
        "engine": (f"autotuned: {r['tuning']['engine']} engine, {r['tuning']['batch']} consecutive windows "
                   "per launch, graph replay (router on when the window engine runs)"),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback",
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": "profiles/ncu_traffic.txt: dram__bytes_read.sum + dram__bytes_write.sum "
                                       "per launch from the committed ncu capture of this kernel on this workload",
                     "algorithmic_bytes_per_launch": slide_bytes * per_launch, "windows_per_launch": per_launch,
                     "algorithmic_bytes_per_slide": slide_bytes,
                     # the dominant kernel's own minimum bytes (its counted points; candidate reads,
                     # shared per group, not included): what the ncu traffic is compared with
                     "kernel_min_bytes_per_launch": alg * per_launch,
                     "launch_ms": launch_ms, "used_bins": ub,
                     "stage_ms_per_slide": prof,
                     # the whole pass against the per-slide bytes of a detector that
                     # reads every window point once per slide: 4dS in + 4dS ring
                     # write + 4dW window read + 4 n_out IDs
                     "pass": pass_roofline(w, n_out, us_slide, peak)},
        "clocks": r["clocks"],
        "gpu_launches": r["launches"],
        "e2e": {"value": world * r["e2e_steps"] * slides * w.slide / r["e2e_s"], "unit": UNIT,
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                "us_per_slide": r["e2e_s"] / (r["e2e_steps"] * slides) * 1e6},
        "outliers_per_slide": n_out, "undetermined_per_slide": r["undet"],
        "router": r.get("router"),
        "tuning": r.get("tuning"),
        "engines": {name: {"us_per_slide": e["dev_ms"] * 1e3 / (e["steps"] * slides),
                           "points_per_s": world * e["steps"] * slides * w.slide / (e["dev_ms"] / 1e3),
                           "gpu_launches_per_step": e["launches"] / e["steps"]}
                    for name, e in res.items()},
        "bit_exact_across_engines": True,
        "streaming": r.get("streaming"),
        "batched": r.get("batched"),
        "router_ab": r.get("router_ab"),
    }
    if not args.no_cpu_baseline and world == 1:
        cb, (coff, cids) = cpu_baseline(w)
        cb["same_outliers_as_gpu"] = bool(np.array_equal(coff, r["offsets"]) and np.array_equal(cids, r["ids"]))
        line["cpu_baseline"] = cb
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement of RTOD's path, all host threads
# ---------------------------------------------------------------------------
def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle
    oracle.build()
    w = workload()
    threads = os.cpu_count() or 1
    for _ in range(max(1, args.warmup)):
        oracle.detect(w.points, w.window, w.slide, w.R, w.K, engine="grid", threads=threads)
    steps = max(1, args.steps)
    t = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        off, _, _ = oracle.detect(w.points, w.window, w.slide, w.R, w.K, engine="grid", threads=threads)
        t += time.perf_counter() - t0
    slides = len(off) - 1
    value = steps * slides * w.slide / t
    sample = (f"{steps} pass(es) over the whole stream ({slides} slides each), CPU restatement of "
              f"RTOD's grid filter + exact count, slides split over {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": t / steps * 1e3,
        "us_per_slide": t / (steps * slides) * 1e6, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded stand-in for RTOD's STK stream)",
        "config": workload_config(w),
        "engine": ("reference CPU path: the oracle's restatement of RTOD's grid filter + exact count "
                   "(pinned to RTOD's own host code; RTOD's GPU path needs OptiX + RT cores)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ncu_case(args, local):
    """Profiler pass of the headline workload with the settings the autotuner
    picks on it in plain runs (span engine, 3 cells per R, 4-warp count
    blocks, up to 256 windows per launch; under ncu the tuner's own timings
    would be distorted): one pass outside the profiler range, then two
    passes inside it (cudaProfilerStart/Stop: run ncu with
    --profile-from-start off)."""
    import torch
    from rtod_b200 import Detector
    w = workload()
    torch.cuda.set_device(local)
    pts = torch.from_numpy(w.points).to(f"cuda:{local}")
    with Detector(w.window, w.slide, w.R, w.K, dim=w.dim, device=local, engine="span", cells_per_r=3,
                  block_warps=4, batch=256) as det:
        r = det.run(pts)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        for _ in range(2):
            det.reset()
            r = det.run(pts)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        tuning = det.tuning
    print(json.dumps({"mode": "ncu", "slides": r.slides, "outliers": int(r.offsets[-1]), "tuning": tuning}))


def run_ncu_stream(args, local, slides: int = 30, engine: str = "window"):
    """Profiler pass of RTOD's per-slide loop on the headline workload
    (push S points from host memory, detect): 10 slides outside the profiler
    range, then `slides` slides inside it (cudaProfilerStart/Stop: run ncu
    with --profile-from-start off)."""
    import torch
    from rtod_b200 import Detector
    w = workload()
    torch.cuda.set_device(local)
    W, S = w.window, w.slide
    with Detector(W, S, w.R, w.K, dim=w.dim, device=local, engine=engine) as det:
        det.push(w.points[:W])
        n_out = 0
        for j in range(10 + slides):
            if j == 10:
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
            det.push(w.points[W + j * S:W + (j + 1) * S])
            n_out += len(det.detect())
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        info = det.stream_engine
    print(json.dumps({"mode": "ncu-stream", "slides": slides, "outliers": n_out, "engine": info["engine"]}))


def run_ncu_batched(args, local, steps: int = 2):
    """Profiler pass of the 8-d streams of the 64-stream workload (26
    streams, W from 5k to 169k, default settings: group counts): two
    multi-stream steps outside the profiler range, then `steps` steps inside
    it (cudaProfilerStart/Stop: run ncu with --profile-from-start off)."""
    import torch
    from rtod_b200 import BatchDetector, datagen
    d8 = [s for s in datagen.batched_streams(slides=2 + steps) if s.dim == 8]
    cfg = [dict(window=s.window, slide=s.slide, R=s.R, K=s.K, dim=s.dim) for s in d8]
    n_out = 0
    with BatchDetector(cfg, device=local) as bd:
        for i, s in enumerate(d8):
            bd.push(i, s.points[:s.window])
        for j in range(2 + steps):
            if j == 2:
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
            for i, s in enumerate(d8):
                bd.push(i, s.points[s.window + j * s.slide:s.window + (j + 1) * s.slide])
            n_out += sum(len(o) for o in bd.step())
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        tuning = bd.tuning
    print(json.dumps({"mode": "ncu-batched", "streams": len(d8), "steps": steps, "outliers": n_out,
                      "tuning": tuning}))


def run_replica_check(world, rank):
    """The replica path of this file on host ranks (gloo): every rank detects
    the same slides of the small random walk with the oracle (the CPU
    restatement), the time is the maximum over ranks, the value counts the
    points of all ranks, the outliers must agree on every rank, and rank 0
    alone prints."""
    from oracle import oracle
    from rtod_b200 import datagen
    ranks = Ranks(world, "gloo", "cpu")
    w = datagen.small_walk()
    slides = 20
    ranks.barrier()
    t0 = time.perf_counter()
    off, ids, _ = oracle.detect(w.points[:w.window + slides * w.slide], w.window, w.slide, w.R, w.K,
                                engine="grid")
    dt = ranks.reduce(time.perf_counter() - t0, "max")
    ranks.barrier()
    digest = float(np.sum(ids * 2654435761 % 1000003)) + float(off[-1]) * 1e6
    same = ranks.reduce(digest, "max") == ranks.reduce(digest, "min")
    ranks.close()
    if rank == 0:
        print(json.dumps({"mode": "replica-check", "n_ranks": world, "slides": slides,
                          "value": world * slides * w.slide / dt, "unit": UNIT, "s_max": dt,
                          "outliers": int(off[-1]), "identical_on_all_ranks": same}))


def main():
    args = parse_args()
    world, rank, local = dist_env()
    if args.mode == "ncu":
        run_ncu_case(args, local)
        return
    if args.mode in ("ncu-stream", "ncu-stream-grid"):
        run_ncu_stream(args, local, engine="grid" if args.mode == "ncu-stream-grid" else "window")
        return
    if args.mode == "ncu-batched":
        run_ncu_batched(args, local)
        return
    if args.mode == "replica-check":
        run_replica_check(world, rank)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    out = run_ours(args, world, rank, local)
    if out is not None:
        w, res = out
        emit_ours(args, world, w, res)


if __name__ == "__main__":
    main()
