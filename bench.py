#!/usr/bin/env python
"""Throughput benchmark of the radiance path: Msamples/s (W*H*spp per
second of render, the reference CLI's metric, src/main.zig:243-264).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

One step renders one frame of the workload.  ``value`` is measured with the
scene resident in HBM and the frame written to device memory (CUDA events on
the launching stream, L2 flushed by a 256 MB write before every step, max
over ranks); ``e2e`` goes through the public C-ABI call with host buffers
(scene upload from pinned memory, render, framebuffer read-back).  Under
torchrun every rank renders its own frame (seed = rank): the work is
sharded by frame with no collective on the data path (weak scaling).

``--impl reference`` times the CPU restatement of the reference renderer
(oracle/, f64, all host threads, same atomic tile scheduler) on a bounded
random sample of the workload's pixels, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FP64_LANES_PER_SM = 64
NOMINAL_SM_MHZ = 1965.0
# DRAM bytes (read + write) per sample of the megakernel, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, one 8-spp launch of the
# workload, --clock-control none) and scaled by samples per launch: traffic
# grows with the samples traced.  Keyed by (workload, precision); workloads
# without a capture report null.
NCU_DRAM_BYTES_PER_SAMPLE = {("triangle_heavy", "exact"): 2.527835e9 / (1920 * 1080 * 8),
                             ("triangle_heavy", "fast"): (1.308102e9 + 1.654117e9) / (1920 * 1080 * 8)}
# What bounds the kernel instead of a pipe peak, from the same capture:
# issue slots used, lanes active per warp instruction, FP64 pipe activity.
NCU_EXECUTION = {("triangle_heavy", "exact"): {"issue_active_pct": 62.7, "lanes_per_warp_instruction": 8.27,
                                               "fp64_pipe_active_pct": 45.9, "l1_hit_pct": 72.2, "l2_hit_pct": 84.3},
                 ("triangle_heavy", "fast"): {"issue_active_pct": 59.5, "lanes_per_warp_instruction": 7.19,
                                              "fp64_pipe_active_pct": 31.5, "fma_pipe_active_pct": 8.7,
                                              "l1_hit_pct": 75.9, "l2_hit_pct": 83.1,
                                              "top_stall": "long_scoreboard 5.4 cycles per issue"},
                 ("batch", "exact"): {"issue_active_pct": 70.2, "lanes_per_warp_instruction": 14.23,
                                      "fp64_pipe_active_pct": 44.5, "l1_hit_pct": 82.9, "l2_hit_pct": 88.5},
                 ("batch", "fast"): {"issue_active_pct": 72.9, "lanes_per_warp_instruction": 14.32,
                                     "fp64_pipe_active_pct": 25.6, "fma_pipe_active_pct": 16.0, "l1_hit_pct": 78.7,
                                     "l2_hit_pct": 88.9, "top_stall": "long_scoreboard 2.9 cycles per issue"}}
# The batched launch, captured whole (rank 0's batch, one launch), by precision.
NCU_DRAM_BYTES_BATCH = {"exact": 0.160607e9 + 1.138117e9, "fast": 0.167182e9 + 2.485141e9}


FP32_LANES_PER_SM = 128


def roofline_entry(work: dict, samples: int, kernel_ms: float, sms: int, traffic, traffic_note: str,
                   execution) -> dict:
    """The roofline object for one kernel: oracle-counted FLOP and bytes per
    sample times the samples of one launch, over its CUDA-event duration.
    When part of the arithmetic is single precision (the fast traversal's box
    tests, work["flop_f32"]), each part is set against its own pipe's peak and
    frac is the share of the kernel's time that the arithmetic would take at
    those peaks (f64 time + f32 time over kernel time)."""
    flop = work["flop"] * samples
    f32 = work.get("flop_f32", 0.0) * samples
    achieved = flop / (kernel_ms / 1e3) / 1e12
    peak = sms * FP64_LANES_PER_SM * 2 * NOMINAL_SM_MHZ * 1e6 / 1e12
    peak32 = sms * FP32_LANES_PER_SM * 2 * NOMINAL_SM_MHZ * 1e6 / 1e12
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    bytes_per_launch = work["bytes"] * samples
    mixed = {}
    peak_used = peak
    if f32 > 0:
        # the rate this mix of f64 and f32 work would reach with each part at
        # its own pipe's peak; achieved / that = the time-weighted fraction
        peak_used = flop / ((flop - f32) / peak + f32 / peak32)
        mixed = {"bound": "fp64+fp32",
                 "split": {"fp64_tflops": round((flop - f32) / (kernel_ms / 1e3) / 1e12, 3),
                           "fp64_peak": round(peak, 1),
                           "fp32_tflops": round(f32 / (kernel_ms / 1e3) / 1e12, 3), "fp32_peak": round(peak32, 1),
                           "note": "box tests in f32 (FMA) against the nominal FP32 peak, primitives and shading "
                                   "in f64 against the nominal FP64 peak; peak = the rate of this mix with each "
                                   "part at its pipe's peak, so frac = the time the arithmetic needs at those "
                                   "peaks over the kernel's time"}}
    return {
        "bound": "fp64", "achieved": round(achieved, 3), "peak": round(peak_used, 1), "unit": "TFLOP/s",
        "frac": round(achieved / peak_used, 4),
        **mixed,
        "traffic": traffic, "traffic_note": traffic_note, "ncu_execution": execution,
        "peak_source": f"nominal FP64: {sms} SMs x 64 lanes x 2 FLOP (FMA) x 1965 MHz; "
                       "no measured FP64 figure exists (the path uses no FMA: its issue-rate ceiling is half)",
        "algorithmic_flop_per_sample": round(work["flop"], 1),
        "algorithmic_bytes_per_sample": round(work["bytes"], 1),
        "kernel_ms": round(kernel_ms, 3),
        "memory": {"achieved_gbs": round(bytes_per_launch / (kernel_ms / 1e3) / 1e9, 1), "peak_gbs": hbm,
                   "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650",
                   "note": "bytes requested from the memory system; most are served by L2"},
        "per_sample": {k: round(v, 3) for k, v in work.items() if k not in ("flop", "bytes", "flop_f32")},
    }


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--workload", default="triangle_heavy",
                   choices=["triangle_heavy", "random_spheres", "cornell", "batch", "diff"])
    p.add_argument("--gd-steps", type=int, default=100, help="gradient-descent steps (--workload diff)")
    p.add_argument("--spp", type=int, default=0, help="override spp (profiling runs)")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample size in seconds")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", dest="autotune", action="store_false",
                   help="use --mode as given instead of the autotuner's choice")
    p.add_argument("--no-extras", action="store_true",
                   help="default workload only: skip the batch and diff sub-objects")
    p.add_argument("--mode", type=int, default=0, help="zt_gpu_config.mode")
    p.add_argument("--capacity", type=int, default=0, help="zt_gpu_config.queue_capacity (wavefront)")
    p.add_argument("--shard", choices=["frames", "rows"], default="frames",
                   help="frames: one frame per rank (weak scaling); rows: one frame split into row bands across "
                        "ranks and all-gathered on the device (strong scaling)")
    p.add_argument("--precision", choices=["exact", "fast"], default="fast",
                   help="zt_gpu_config.precision of the measured render (exact = the verification build)")
    return p.parse_args()


def workload(name: str, spp_override: int):
    import zigtrace_b200 as zt
    from zigtrace_b200 import scenes
    build, opts = scenes.WORKLOADS[name]
    scene = build()
    o = zt.Options(**{k: getattr(opts, k) for k in ("width", "height", "spp", "max_depth", "seed")})
    if spp_override:
        o.spp = spp_override
    return scene, o


def describe(name, scene, o, counts):
    desc = {
        "triangle_heavy": "1M-triangle heightfield + 20 icospheres + 64 emissive quads, NEE+MIS",
        "random_spheres": "random spheres (ground plane + ~320 spheres, thin lens), no emitters",
        "cornell": "Cornell box (glass + metal sphere, ceiling area light), NEE+MIS",
    }[name]
    return {"workload": f"{name}: {desc}, {o.width}x{o.height}, {o.spp} spp, depth {o.max_depth}",
            "width": o.width, "height": o.height, "spp": o.spp, "max_depth": o.max_depth,
            "bounded_primitives": counts["bounded"], "planes": counts["planes"], "bvh_nodes": counts["nodes"],
            "sampled_lights": counts["lights"]}


# ------------------------------------------------------------- CPU leg ----
def measured_image_error(scene, o, img, threads: int, n_pixels: int = 4000, rng_seed: int = 11) -> dict:
    """The measured frame against the oracle at the same seed on random
    pixels: per-channel relative RMSE and mean luminance in Monte Carlo
    standard errors (oracle/agreement.py)."""
    import numpy as np
    import oracle as O
    from oracle.agreement import image_agreement
    rng = np.random.default_rng(rng_seed)
    pix = np.unique(rng.integers(0, o.width * o.height, n_pixels)).astype(np.uint64)
    want, m2 = O.OracleScene.from_scene(scene).render_pixels_moments(o.width, o.height, o.spp, o.max_depth, pix,
                                                                     threads=threads, seed=o.seed,
                                                                     light_sampling=o.light_sampling)
    a = image_agreement(img.reshape(-1, 3)[pix.astype(np.int64)], want, m2, o.spp)
    a["pixels"] = int(len(pix))
    return a


def cpu_sample(scene, o, seconds: float, threads: int, rng_seed: int = 1, oscene=None):
    """Oracle render of random pixels of the workload, sized to ~seconds."""
    import numpy as np
    import oracle as O
    os_ = oscene if oscene is not None else O.OracleScene.from_scene(scene)
    npix = o.width * o.height
    rng = np.random.default_rng(rng_seed)
    n = 64
    while True:
        pix = np.sort(rng.choice(npix, size=min(n, npix), replace=False)).astype(np.uint64)
        t0 = time.perf_counter()
        _, st = os_.render_pixels(o.width, o.height, o.spp, o.max_depth, pix, threads=threads, seed=o.seed,
                                  light_sampling=o.light_sampling, stats=True)
        dt = time.perf_counter() - t0
        if dt >= 0.8 * seconds or n >= npix:
            return len(pix), dt, st
        n = int(min(npix, max(n * 2, n * seconds / max(dt, 1e-3) * 1.05)))


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    scene, o = workload(args.workload, args.spp)  # NumPy arrays only: the product library is never loaded
    import numpy as np
    import oracle as O
    os_ = O.OracleScene.from_scene(scene)
    counts_scene = os_.counts()
    per_step = max(args.cpu_seconds / 3.0, 2.0)
    n_pix, _, _ = cpu_sample(scene, o, per_step, threads, oscene=os_)  # calibration
    rng = np.random.default_rng(7)
    times = []
    for i in range(args.warmup + args.steps):
        pix = np.sort(rng.choice(o.width * o.height, size=n_pix, replace=False)).astype(np.uint64)
        t0 = time.perf_counter()
        os_.render_pixels(o.width, o.height, o.spp, o.max_depth, pix, threads=threads, seed=o.seed)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    samples = n_pix * o.spp
    value = samples / statistics.mean(times) / 1e6
    sample_desc = f"{n_pix} random pixels x {o.spp} spp ({samples} samples) per step"
    emit({
        "impl": "reference", "metric": "Msamples/s", "value": round(value, 4), "unit": "Msamples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * statistics.mean(times), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural scene)",
        "config": describe(args.workload, scene, o, counts_scene),
        "cpu_baseline": {"value": round(value, 4), "unit": "Msamples/s", "cores": threads, "kind": "port",
                         "sample": sample_desc + "; C restatement of the reference CPU renderer (oracle/), "
                                                 "-O3 -ffp-contract=off, atomic tile scheduler"},
        "e2e": {"value": round(value, 4), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })


# -------------------------------------------------------------- clocks ----
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        self.gpu = ids[local_rank] if local_rank < len(ids) else str(local_rank)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.gpu], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [[c.strip() for c in line.split(",")] for line in out.splitlines() if line.count(",") >= 8]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------- GPU leg ----
def e2e_breakdown(scene, o, gcfg, d_out, pinned, args, allmax) -> dict:
    """Where an end-to-end step's time goes: the same work as separate public
    calls, each timed on the host after a device synchronisation -- scene
    upload (device allocation from the library's pool + host-to-device copy),
    render into device memory, framebuffer read-back into pinned memory."""
    import torch

    import zigtrace_b200 as zt
    up, rend, back = [], [], []
    for i in range(args.warmup + args.steps):
        scene.release_device()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scene.upload()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        zt.render_device(scene, o, d_out.data_ptr(), 0, gcfg)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        pinned.copy_(d_out)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        if i >= args.warmup:
            up.append(t1 - t0)
            rend.append(t2 - t1)
            back.append(t3 - t2)
    return {"upload": round(1e3 * allmax(statistics.mean(up)), 3),
            "render": round(1e3 * allmax(statistics.mean(rend)), 3),
            "readback": round(1e3 * allmax(statistics.mean(back)), 3)}


def b200_arm(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import zigtrace_b200 as zt
    from zigtrace_b200 import _native as N
    from zigtrace_b200 import workmodel

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1 or args.shard == "rows":
        from datetime import timedelta
        if "MASTER_ADDR" not in os.environ:  # a single-rank group for the row-sharded mode at N=1
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(29500 + os.getpid() % 1000), RANK="0",
                              WORLD_SIZE="1")
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local_rank))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.shard == "rows":
        line = shard_rows_arm(args, world, rank, local_rank, barrier, allmax)
        if rank == 0:
            emit(line)
        dist.destroy_process_group()
        return
    if args.workload in ("batch", "diff"):
        arm = batch_arm if args.workload == "batch" else diff_arm
        line = arm(args, world, rank, local_rank, barrier, allmax)
        if rank == 0:
            emit(line)
        if world > 1:
            dist.destroy_process_group()
        return
    scene, o = workload(args.workload, args.spp)
    o.seed = o.seed + rank  # each rank renders its own frame
    scene.build(device=True)  # the same tree as the host build (zt_scene_build_device)
    counts = scene.counts()
    scene.upload()
    prec = zt.PRECISION_FAST if args.precision == "fast" else zt.PRECISION_EXACT
    gcfg = zt.GpuConfig(mode=args.mode, queue_capacity=args.capacity, precision=prec)
    tuned = None
    if args.autotune:  # mode, block size and queue capacity from the project's autotuner
        from zigtrace_b200 import autotune
        gcfg, tune_ms, tune_cached = autotune.tune_render(scene, o, reps=1, precision=prec)
        tuned = {"mode": ["auto", "megakernel", "wavefront", "megakernel_regen", "wavefront_sorted"][gcfg.mode],
                 "block_size": gcfg.block_size, "queue_capacity": gcfg.queue_capacity, "precision": args.precision,
                 "cached": tune_cached, "candidates_ms": tune_ms,
                 "candidate_key": "[mode, block_size, queue_capacity]"}
    npix = o.width * o.height
    samples = npix * o.spp
    out = torch.empty(npix * 3, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream()

    def step():
        flush.zero_()
        zt.render_device(scene, o, out.data_ptr(), stream.cuda_stream, gcfg)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    k_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    k_end = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_start.record(stream)
    for i in range(args.steps):
        flush.zero_()
        k_start[i].record(stream)
        zt.render_device(scene, o, out.data_ptr(), stream.cuda_stream, gcfg)
        k_end[i].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    elapsed_ms = allmax(t_start.elapsed_time(t_end))
    kernel_ms = allmax(statistics.mean(k_start[i].elapsed_time(k_end[i]) for i in range(args.steps)))
    ms_per_step = elapsed_ms / args.steps
    value = world * samples / (ms_per_step / 1e3) / 1e6
    img = out.cpu().numpy()
    assert np.isfinite(img).all(), "non-finite pixel in the framebuffer"

    verification = None
    if prec == zt.PRECISION_FAST and not args.no_extras:
        # the verification build (bit-identical to the reference algorithm) on
        # the same frame, timed the same way
        vcfg = zt.GpuConfig(mode=gcfg.mode, block_size=gcfg.block_size, queue_capacity=gcfg.queue_capacity,
                            precision=zt.PRECISION_EXACT)
        for _ in range(args.warmup):
            flush.zero_()
            zt.render_device(scene, o, out.data_ptr(), stream.cuda_stream, vcfg)
        torch.cuda.synchronize()
        barrier()
        v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        v0.record(stream)
        for _ in range(args.steps):
            flush.zero_()
            zt.render_device(scene, o, out.data_ptr(), stream.cuda_stream, vcfg)
        v1.record(stream)
        torch.cuda.synchronize()
        barrier()
        v_ms = allmax(v0.elapsed_time(v1)) / args.steps
        exact_img = out.cpu().numpy()
        verification = {"precision": "exact", "value": round(world * samples / (v_ms / 1e3) / 1e6, 4),
                        "unit": "Msamples/s", "ms_per_step": round(v_ms, 3),
                        "fast_over_exact": round(v_ms / ms_per_step, 3),
                        "identical_pixels_fast_vs_exact": float((exact_img.reshape(-1, 3) ==
                                                                 img.reshape(-1, 3)).all(axis=1).mean())}

    # ---- e2e through the public C-ABI call with host buffers
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(npix * 3, dtype=torch.float64).pin_memory()
        rec = o.record()
        times = []
        for i in range(args.warmup + args.steps):
            scene.release_device()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            N.check(N.lib().zt_render_ex(scene.handle, N.ptr(rec), N.ptr(gcfg.record()),
                                         __import__("ctypes").c_void_p(pinned.data_ptr())))
            t1 = time.perf_counter()
            if i >= args.warmup:
                times.append(t1 - t0)
        e2e_s = allmax(statistics.mean(times))
        e2e = {"value": round(world * samples / e2e_s / 1e6, 4), "unit": "Msamples/s",
               "h2d_bytes_per_step": scene.staging_bytes(), "d2h_bytes_per_step": npix * 3 * 8,
               "ms_per_step": round(1e3 * e2e_s, 3), "host_buffers": "pinned",
               "breakdown_ms": e2e_breakdown(scene, o, gcfg, out, pinned, args, allmax),
               "identical_to_device_arm": bool((pinned.numpy() == img).all())}
        e2e["breakdown_ms"]["unaccounted"] = round(1e3 * e2e_s - sum(e2e["breakdown_ms"].values()), 3)
        scene.upload()

    # ---- CPU baseline and per-sample work from the oracle (rank 0, N=1)
    cpu = None
    work = None
    queue_bytes = None
    image_error = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        n_pix, dt, st = cpu_sample(scene, o, args.cpu_seconds, threads)
        cpu = {"value": round(n_pix * o.spp / dt / 1e6, 4), "unit": "Msamples/s", "cores": threads, "kind": "port",
               "sample": f"{n_pix} random pixels x {o.spp} spp ({n_pix * o.spp} samples), oracle C restatement "
                         f"of the reference CPU renderer, {threads} threads, {dt:.1f} s"}
        work = workmodel.per_sample(st, o.spp, counts["nodes"] > 0, fast=prec == zt.PRECISION_FAST)
        queue_bytes = workmodel.wavefront_queue_bytes(st, o.spp)
        image_error = measured_image_error(scene, o, img, threads)

    roofline = None
    if work is not None:
        sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
        roofline = roofline_entry(
            work, samples, kernel_ms, sms,
            (round(NCU_DRAM_BYTES_PER_SAMPLE[(args.workload, args.precision)] * samples)
             if (args.workload, args.precision) in NCU_DRAM_BYTES_PER_SAMPLE and gcfg.mode in (0, 1) else None),
            "DRAM bytes per launch from an ncu capture of an 8-spp launch, scaled by samples",
            NCU_EXECUTION.get((args.workload, args.precision)) if gcfg.mode in (0, 1) else None)
        if gcfg.mode in (2, 4):  # the wavefront form: path-state traffic through HBM against the copy peak
            qbps = queue_bytes * samples / (kernel_ms / 1e3) / 1e9
            roofline["queue"] = {"bytes_per_sample": round(queue_bytes, 1), "achieved_gbs": round(qbps, 1),
                                 "peak_gbs": roofline["memory"]["peak_gbs"],
                                 "frac": round(qbps / roofline["memory"]["peak_gbs"], 4),
                                 "note": "path-state bytes of the wavefront kernels (workmodel.py), "
                                         "oracle-counted rays, hits and shadow rays per sample"}

    line = {
        "metric": "Msamples/s", "value": round(value, 4), "unit": "Msamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural scene)",
        "config": {**describe(args.workload, scene, o, counts), "l2": "flushed by a 256 MB write before every step",
                   "mode": ["auto", "megakernel", "wavefront", "megakernel_regen", "wavefront_sorted"][gcfg.mode],
                   "precision": args.precision, "autotune": tuned,
                   "sharding": "one frame per rank (seed = rank), no collective",
                   "bvh_build": {"on_device": scene.built_on_device,
                                 "device_ms": round(scene.build_ms, 2) if scene.build_ms else None}},
        "e2e": e2e, "gpu_launches": args.steps, "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
        "image_error": image_error, "verification_build": verification,
    }
    if not args.no_extras:
        # the other two parts of the metric, each with its own clocks, e2e and
        # timing: batched vs plain launches, and backward vs forward time
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup, sub.spp = min(args.steps, 10), 3, 0
        del out, flush
        torch.cuda.empty_cache()
        line["diff"] = diff_arm(sub, world, rank, local_rank, barrier, allmax)  # host-timed: before the batch's load
        torch.cuda.empty_cache()
        line["batch"] = batch_arm(sub, world, rank, local_rank, barrier, allmax)
    if rank == 0:
        emit(line)
    if world > 1:
        dist.destroy_process_group()


def shard_rows_arm(args, world, rank, local_rank, barrier, allmax):
    """One frame of the workload split into row bands across the ranks: each
    rank renders its band into its slot of a device buffer
    (zt_render_rows_device) and one NCCL all-gather assembles the frame on
    every rank, inside the timed region.  value = the frame's samples over
    the max-over-ranks time per frame (strong scaling: the frame is fixed)."""
    import torch
    import torch.distributed as dist

    import zigtrace_b200 as zt
    from zigtrace_b200 import sharding

    scene, o = workload(args.workload, args.spp)
    scene.build(device=True)
    scene.upload()
    prec = zt.PRECISION_FAST if args.precision == "fast" else zt.PRECISION_EXACT
    gcfg = zt.GpuConfig(mode=args.mode, precision=prec)
    height, width = int(o.height), int(o.width)
    bands = sharding.row_bands(height, world)
    y0, y1 = bands[rank]
    max_rows = max(b - a for a, b in bands)
    buf = torch.zeros(max_rows * width * 3, dtype=torch.float64, device="cuda")
    gathered = torch.empty(world * buf.numel(), dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        zt.render_rows_device(scene, o, y0, y1, buf.data_ptr(), stream.cuda_stream, gcfg)
        dist.all_gather_into_tensor(gathered, buf)

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    k1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    a.record(stream)
    for i in range(args.steps):
        flush.zero_()
        k0[i].record(stream)
        step()
        k1[i].record(stream)
    b.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = allmax(a.elapsed_time(b)) / args.steps
    frame_ms = allmax(statistics.mean(k0[i].elapsed_time(k1[i]) for i in range(args.steps)))
    samples = width * height * o.spp
    stride = buf.numel()
    img = torch.cat([gathered[r * stride:r * stride + (q - p) * width * 3] for r, (p, q) in enumerate(bands)])
    whole = torch.empty(width * height * 3, dtype=torch.float64, device="cuda")
    zt.render_device(scene, o, whole.data_ptr(), stream.cuda_stream, gcfg)
    torch.cuda.synchronize()
    identical = bool(torch.equal(img, whole))
    counts = scene.counts()
    return {
        "metric": "Msamples/s", "value": round(samples / (ms / 1e3) / 1e6, 4), "unit": "Msamples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded procedural scene)",
        "config": {**describe(args.workload, scene, o, counts), "l2": "flushed by a 256 MB write before every step",
                   "precision": args.precision,
                   "sharding": f"one frame in {world} row bands (rows {bands}), band rendered into its slot of "
                               "the gather buffer, one NCCL all-gather per frame inside the timed region"},
        "frame_ms_with_gather": round(frame_ms, 3), "gathered_equals_single_device_render": identical,
        "gpu_launches": args.steps, "clocks": clk, "roofline": None, "cpu_baseline": None,
        "e2e": None,
    }


def batch_arm(args, world, rank, local_rank, barrier, allmax):
    """The batched form: 256 sphere-field renders (16..20000 spheres, 64^2..512x288,
    16 spp, depth 16) in one persistent launch replayed from a CUDA graph,
    against the same 256 renders as plain per-scene launches."""
    import numpy as np
    import torch
    import torch.distributed as dist

    import zigtrace_b200 as zt
    from zigtrace_b200 import autotune, scenes

    items = scenes.batch_workload(seed=1000 * rank)  # each rank its own batch
    scs, opts = [s for s, _ in items], [o for _, o in items]
    for s in scs:
        s.build()
        s.upload()
    samples = sum(o.width * o.height * o.spp for o in opts)
    outs = [torch.empty(o.width * o.height * 3, dtype=torch.float64, device="cuda") for o in opts]
    prec = zt.PRECISION_FAST if args.precision == "fast" else zt.PRECISION_EXACT
    cfg, order, tune_ms, cached = autotune.tune_batch(scs, opts, reps=1, precision=prec)
    plain_won = order == autotune.PLAIN
    if plain_won:  # still measure the best batched launch against the plain launches
        best = json.loads(min((k for k in tune_ms if json.loads(k)[0] != autotune.PLAIN), key=tune_ms.get))
        cfg, order = zt.GpuConfig(mode=best[2], block_size=best[0], precision=prec), best[1]
    batch = zt.Batch(scs, opts, [t.data_ptr() for t in outs], cfg, order)
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def plain():
        for s, o, t in zip(scs, opts, outs):
            zt.render_device(s, o, t.data_ptr(), stream.cuda_stream, zt.GpuConfig(precision=prec))

    def timed(fn):
        for _ in range(args.warmup):
            flush.zero_()
            fn()
        torch.cuda.synchronize()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            flush.zero_()
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        barrier()
        return allmax(a.elapsed_time(b)) / args.steps

    clocks = ClockSampler(local_rank)
    clocks.start()
    batch_ms = timed(lambda: batch.launch(stream.cuda_stream))
    clk = clocks.stop()
    batched_imgs = [t.cpu() for t in outs]
    plain_ms = timed(plain)
    same = all(torch.equal(x, t.cpu()) for x, t in zip(batched_imgs, outs))
    value = world * samples / (batch_ms / 1e3) / 1e6
    plain_value = world * samples / (plain_ms / 1e3) / 1e6

    e2e = None
    if not args.no_e2e:  # zt_render_batch into pinned host buffers, scenes re-uploaded every step
        import ctypes as C
        from zigtrace_b200 import _native as N
        pinned = [torch.empty(o.width * o.height * 3, dtype=torch.float64).pin_memory() for o in opts]
        handles = (C.c_void_p * len(scs))(*[s.handle.value for s in scs])
        recs = np.concatenate([o.record() for o in opts])
        ptrs = (C.c_void_p * len(scs))(*[t.data_ptr() for t in pinned])
        bcfg = cfg.record()
        times = []
        for i in range(args.warmup + args.steps):
            for s in scs:
                s.release_device()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            N.check(N.lib().zt_render_batch(handles, N.ptr(recs), len(scs), ptrs, N.ptr(bcfg)))
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
        e2e_s = allmax(statistics.mean(times))
        e2e = {"value": round(world * samples / e2e_s / 1e6, 4), "unit": "Msamples/s",
               "h2d_bytes_per_step": sum(s.staging_bytes() for s in scs),
               "d2h_bytes_per_step": sum(o.width * o.height * 24 for o in opts)}
        same_e2e = all(torch.equal(x, t) for x, t in zip(batched_imgs, pinned))
        times = []  # the same 256 renders as one zt_render_ex call each, into the same pinned buffers
        pcfg = zt.GpuConfig(precision=prec).record()  # each render at the library's default choice
        orecs = [o.record() for o in opts]
        for i in range(args.warmup + args.steps):
            for s in scs:
                s.release_device()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for s, r, t in zip(scs, orecs, pinned):
                N.check(N.lib().zt_render_ex(s.handle, N.ptr(r), N.ptr(pcfg), C.c_void_p(t.data_ptr())))
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
        plain_e2e_s = allmax(statistics.mean(times))
        e2e["plain_calls_value"] = round(world * samples / plain_e2e_s / 1e6, 4)
        e2e["batched_over_plain_calls"] = round(plain_e2e_s / e2e_s, 3)
        e2e["host_buffers"] = "pinned"
        e2e["identical_to_device_arm"] = bool(same_e2e and
                                              all(torch.equal(x, t) for x, t in zip(batched_imgs, pinned)))

    cpu = None
    roofline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle as O
        from zigtrace_b200 import workmodel
        rng = np.random.default_rng(3)
        threads = os.cpu_count() or 1
        n_s, t_s = 0, 0.0
        work_w = {}  # per-sample work of each sampled render, weighted by the render's samples
        weight = 0
        for k in rng.choice(len(items), 32, replace=False):
            s, o = items[int(k)]
            os_ = O.OracleScene.from_scene(s)  # BVH build outside the timed region, as in the reference CLI
            pix = np.sort(rng.choice(o.width * o.height, min(1024, o.width * o.height), replace=False))
            t0 = time.perf_counter()
            _, st = os_.render_pixels(o.width, o.height, o.spp, o.max_depth, pix.astype(np.uint64), threads=threads,
                                      stats=True)
            t_s += time.perf_counter() - t0
            n_s += len(pix) * o.spp
            w = o.width * o.height * o.spp
            for key, v in workmodel.per_sample(st, o.spp, fast=prec == zt.PRECISION_FAST).items():
                work_w[key] = work_w.get(key, 0.0) + v * w
            weight += w
        cpu = {"value": round(n_s / t_s / 1e6, 4), "unit": "Msamples/s", "cores": threads, "kind": "port",
               "sample": f"1024 random pixels x 16 spp from each of 32 random renders of the batch ({n_s} samples)"}
        sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
        roofline = roofline_entry(
            {key: v / weight for key, v in work_w.items()}, samples, batch_ms, sms,
            round(NCU_DRAM_BYTES_BATCH[args.precision]),
            "DRAM bytes of one batched launch of this batch (seed 0), from an ncu capture",
            NCU_EXECUTION.get(("batch", args.precision)))
        roofline["work_note"] = ("per-sample work averaged over 32 sampled renders, each weighted by its samples "
                                 "per step")

    line = {
        "metric": "Msamples/s", "value": round(value, 4), "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(batch_ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural scenes)",
        "config": {"workload": "batch: 256 sphere-field renders, sphere count log-uniform in [16, 20000], "
                               "resolution from {64x64, 128x128, 256x256, 512x288}, 16 spp, depth 16, NEE on",
                   "renders": len(items), "samples_per_step": samples,
                   "l2": "flushed by a 256 MB write before every step",
                   "precision": args.precision,
                   "autotune": {"block_size": cfg.block_size, "order": ["given", "largest_first"][order],
                                "mode": ["auto", "megakernel", "wavefront", "megakernel_regen"][cfg.mode],
                                "plain_launches_won": plain_won, "cached": cached, "candidates_ms": tune_ms,
                                "candidate_key": "[block_size, order, mode]; [-1, 0, 1] = plain per-render launches"},
                   "sharding": "one batch per rank (seeds offset by rank), no collective"},
        "plain_launches": {"value": round(plain_value, 4), "unit": "Msamples/s", "ms_per_step": round(plain_ms, 3),
                           "launches_per_step": len(items)},
        "batched_over_plain": round(plain_ms / batch_ms, 3), "identical_images": bool(same),
        "e2e": e2e, "gpu_launches": args.steps, "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
    }
    batch.close()
    return line


def diff_arm(args, world, rank, local_rank, barrier, allmax):
    """The differentiable form: Cornell-style box with 32 Lambertian albedos
    and 4 emitter radiances as parameters, 512x512, 64 spp, L2 loss against
    a target rendered at parameters perturbed by +/-20%.  Reports forward and
    backward time through zt_forward / zt_backward (host buffers), the
    adjoint against central finite differences with common random numbers
    (h = 1e-3), and a 100-step gradient descent."""
    import numpy as np
    import torch
    import torch.distributed as dist

    import zigtrace_b200 as zt
    from zigtrace_b200 import scenes

    scene, target = scenes.cornell_diff(seed=rank)
    scene.build()
    o = scenes.DIFF_OPTIONS
    if args.spp:
        o = zt.Options(o.width, o.height, args.spp, o.max_depth)
    theta0 = np.array([m["color"] for m in scene.materials])
    target_img = zt.forward(scene, o, target).pixels
    samples = o.width * o.height * o.spp

    def fwd(th):
        return zt.forward(scene, o, th).pixels

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        ts = []
        for _ in range(max(args.steps, 9)):  # host-timed calls: the median of at least 9 resists host jitter
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        barrier()
        return allmax(statistics.median(ts))

    img = fwd(theta0)
    d_img = 2.0 * (img - target_img)
    clocks = ClockSampler(local_rank)
    clocks.start()
    fwd_s = timed(lambda: fwd(theta0))
    bwd_s = timed(lambda: zt.backward(scene, o, d_img, theta0))
    clk = clocks.stop()
    grad = zt.backward(scene, o, d_img, theta0)

    h, errs, fd_vals = 1e-3, [], {}
    for m, c in ((0, 0), (9, 1), (22, 2), (31, 0), (32, 1), (35, 2)):
        tp, tm = theta0.copy(), theta0.copy()
        tp[m, c] += h
        tm[m, c] -= h
        fd = (((fwd(tp) - target_img) ** 2).sum() - ((fwd(tm) - target_img) ** 2).sum()) / (2 * h)
        fd_vals[f"{m},{c}"] = [float(grad[m, c]), float(fd)]
        errs.append(abs(grad[m, c] - fd) / max(abs(fd), 1e-12))

    th = torch.tensor(theta0, dtype=torch.float64)
    albedo, radiance = th[:32].clone().requires_grad_(), th[32:].clone().requires_grad_()
    opt = torch.optim.Adam([{"params": [albedo], "lr": 0.01}, {"params": [radiance], "lr": 0.2}])
    f = zt.render_function()
    tgt = torch.from_numpy(target_img.copy())
    losses = []
    t0 = time.perf_counter()
    for _ in range(args.gd_steps):
        opt.zero_grad()
        loss = ((f.apply(torch.cat([albedo, radiance]), scene, o) - tgt) ** 2).mean()
        loss.backward()
        opt.step()
        with torch.no_grad():
            albedo.clamp_(0.01, 0.99)
            radiance.clamp_(min=0.0)
        losses.append(loss.item())
    gd_s = time.perf_counter() - t0
    final = torch.cat([albedo, radiance]).detach().numpy()
    param_err0 = float(np.abs(theta0 - target).mean())
    param_err = float(np.abs(final - target).mean())

    line = {
        "metric": "Msamples/s", "value": round(world * samples / fwd_s / 1e6, 4), "unit": "Msamples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * fwd_s, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded procedural scene)",
        "config": {"workload": "diff: Cornell-style box, 32 Lambertian albedos + 4 emitter radiances as parameters, "
                               f"{o.width}x{o.height}, {o.spp} spp, depth {o.max_depth}, L2 loss vs a target at "
                               "parameters perturbed by +/-20%", "parameters": int(theta0.size)},
        "forward_ms": round(1e3 * fwd_s, 3), "backward_ms": round(1e3 * bwd_s, 3),
        "backward_over_forward": round(bwd_s / fwd_s, 3),
        "adjoint_vs_fd": {"h": h, "max_rel_err": float(max(errs)), "grad_and_fd": fd_vals},
        "gradient_descent": {"steps": args.gd_steps, "seconds": round(gd_s, 2), "loss_first": losses[0],
                             "loss_last": losses[-1], "mean_abs_param_err_start": param_err0,
                             "mean_abs_param_err_end": param_err},
        "e2e": {"value": round(world * samples / fwd_s / 1e6, 4), "unit": "Msamples/s",
                "h2d_bytes_per_step": int(theta0.nbytes), "d2h_bytes_per_step": o.width * o.height * 24},
        "gpu_launches": args.steps, "clocks": clk, "roofline": None, "cpu_baseline": None,
    }
    return line


def emit(line: dict) -> None:
    """Prints the run's JSON line on the process's original standard output."""
    out = _JSON_OUT if _JSON_OUT is not None else sys.stdout
    print(json.dumps(line), file=out, flush=True)


_JSON_OUT = None


def main():
    global _JSON_OUT
    # Native libraries (NCCL prints a version banner from rank 0 when its
    # first communicator comes up) write to file descriptor 1 directly; the
    # contract is one JSON line on standard output, so descriptor 1 is pointed
    # at standard error for the run and the line goes to a copy of the
    # original.
    sys.stdout.flush()
    saved = os.dup(1)
    _JSON_OUT = os.fdopen(os.dup(saved), "w")
    os.dup2(2, 1)
    try:
        args = parse_args()
        if args.impl == "reference":
            reference_arm(args)
        else:
            b200_arm(args)
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)  # descriptor 1 as the caller had it
        os.close(saved)
        _JSON_OUT.close()
        _JSON_OUT = None


if __name__ == "__main__":
    main()
