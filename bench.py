"""Benchmark: projections/s of the cone-beam forward projector on B200.

Workload (one step): the 256^3 -> 512^2 short-scan configuration -- a 256^3
float32 volume (1 mm voxels, water cylinder + 40 seeded ellipsoids), 360 views
over 200 deg + fan angle, flat 512 x 512 detector at 0.6 mm, SID 750 mm,
SDD 1200 mm, seeded per-view jitter (+-0.5 mm source/detector, +-0.2 deg
tilt), raySampling 0.3, trilinear interpolation, up-sampling 1.  One step
projects all 360 views.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value    views/s over all ranks of the drop-in projector (FP32 storage, default
         settings), volume resident on the device, device-side P matrices and
         output, CUDA-event timed per step (L2 flushed between steps by writing
         a 256 MiB buffer, outside the timed events)
e2e      the same job through the C ABI call a CTL user makes
         (ctlcu_project_volume): host volume, host P matrices, host output,
         copies inside the timed region
roofline the ray-casting kernel's gather bytes (samples x 8 taps x voxel bytes +
         output) per launch over its CUDA-event duration, against on-SM L1
         delivery (SMs x 128 B/clk x sampled SM clock)
legs     (one GPU) the rest of the headline metric on the same workload: the
         batched BF16 form (BF16 storage, 8 requests of 45 views, one CUDA
         graph replay per step: a plan), the plain FP32 gather
         loop it is compared with, the FP64 accumulator, and DRR serving
         latency (8 x 256^3 BF16, Poisson 2000 requests/s)
--impl reference   the reference's own kernel (raycasterprojector_interp.cl
         compiled for the CPU, oracle/_ref) on all host cores, a bounded
         sample of the same views per step
Multi-GPU: one process per GPU (torchrun); the 360 views are split into
contiguous blocks by ctlcu_split_views (the view split of the multi-device
projector), each rank projecting its block with its own copy of the volume:
strong scaling, no data-path collective.
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

VOXEL = (1.0, 1.0, 1.0)
SHAPE = (256, 256, 256)
CHANNELS = ROWS = 512
N_VIEWS = 360
METRIC = "projections/s at 256\u00b3\u2192512\u00b2 (plain FP32 vs batched BF16); p50/p99 DRR latency"
WORKLOAD = "256^3 f32 ellipsoid phantom -> 360 x 512^2 short-scan (200 deg + fan), raySampling 0.3, trilinear"
# DRAM bytes (read + write) of one 360-view launch of the cell loop on this
# workload, from one ncu capture (profiles/cells_kernel_256cubed_to_512sq_dram.md),
# with the launch shape it was captured at (views per block, lanes_x, rays per block, unroll)
# and its accumulator
CELLS_TRAFFIC_BYTES = 7.883831808e9 + 0.424111872e9
CELLS_TRAFFIC_SHAPE = (2, 4, 256, 4)
CELLS_TRAFFIC_ACCUM = "kahan"


def make_inputs(n_views: int = N_VIEWS):
    """The phantom and the 360-view geometry; n_views < 360 takes evenly spaced views
    of the same scan (a small case for profiling)."""
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph
    vol = Ph.ellipsoid_phantom(SHAPE, VOXEL, 40, seed=2)
    det = G.FlatDetector(CHANNELS, ROWS, 0.6, 0.6)
    fan = G.fan_angle(det, 1200.0)
    P = G.circular_flat(N_VIEWS, 750.0, 1200.0, det, angle_range=math.radians(200.0) + fan,
                        rng=np.random.default_rng(2024), jitter_mm=0.5, tilt_deg=0.2)
    if n_views < N_VIEWS:
        P = np.ascontiguousarray(P[np.linspace(0, N_VIEWS - 1, n_views).round().astype(int)])
    return vol, P


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _launched_by_torchrun() -> bool:
    return "TORCHELASTIC_RUN_ID" in os.environ or int(os.environ.get("WORLD_SIZE", "1")) > 1


def dist_setup(n_gpus):
    """One process per GPU.  Under torchrun the NCCL group is made for any world
    size, one rank included, so the barrier and the max over ranks take the same
    NCCL path at every N."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if _launched_by_torchrun():
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def _dist_on() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized()


def max_over_ranks(x: float, world: int) -> float:
    if not _dist_on():
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if _dist_on():
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_rate(vol, P, target_s: float, threads: int):
    """The reference's kernel on the host: time a bounded, evenly spaced view sample."""
    import oracle
    t0 = time.perf_counter()
    oracle.project_ref(vol, VOXEL, P[:1], CHANNELS, ROWS, threads=threads)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(N_VIEWS, round(target_s / max(t1, 1e-3)))))
    idx = np.linspace(0, N_VIEWS - 1, n).round().astype(int)
    t0 = time.perf_counter()
    oracle.project_ref(vol, VOXEL, P[idx], CHANNELS, ROWS, threads=threads)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def bench_config(world: int, n_views: int = N_VIEWS) -> dict:
    """The workload, identical in both arms' lines (what was run, not how it was tuned)."""
    return {"workload": WORKLOAD, "views_per_step": n_views, "volume": "256^3 f32, 1 mm", "detector": "512x512",
            "l2": "flushed between steps (256 MiB write outside the timed events)",
            "parallelism": f"views split over {world} GPU(s) in contiguous blocks (ctlcu_split_views)"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    threads = os.cpu_count() or 1
    line = {"impl": "reference", "metric": METRIC, "unit": "projections/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid phantom, seeded jittered geometry)",
            "config": bench_config(world)}
    if not oracle.ref_available():
        line["unavailable"] = "oracle/_ref/libctlref.so (reference kernel compiled for the CPU) is not built"
        print(json.dumps(line))
        return 0
    vol, P = make_inputs()
    # one step = a bounded sample of views spread over the scan
    per_step = max(1, int(args.ref_views))
    idx = np.linspace(0, N_VIEWS - 1, per_step).round().astype(int)
    for _ in range(args.warmup):
        oracle.project_ref(vol, VOXEL, P[idx[:1]], CHANNELS, ROWS, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.project_ref(vol, VOXEL, P[idx], CHANNELS, ROWS, threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = per_step / (ms / 1e3)
    sample = f"{per_step} of {N_VIEWS} views per step, evenly spaced, {threads} threads"
    line.update({"value": value, "ms_per_step": ms, "scaling": "none",
                 "cpu_baseline": {"value": value, "unit": "projections/s", "cores": threads,
                                  "kind": "reference", "sample": sample},
                 "e2e": {"value": value, "unit": "projections/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0},
                 "vs_baseline": None})
    print(json.dumps(line))
    return 0


def _time_steps(fn, steps, warmup, stream, flush=None):
    """CUDA-event times (ms) of `steps` calls of fn on `stream` after `warmup`
    untimed ones; `flush` (if given) runs between the timed calls, outside the events."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in ev:
        if flush is not None:
            flush()
        a.record(stream)
        fn()
        b.record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def run_ours(args):
    import torch

    import ctl_b200
    from ctl_b200 import _lib as L
    from ctl_b200.projector import Context, Settings, VoxelVolume

    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_views = args.views
    vol, P_all = make_inputs(n_views)
    # this rank's contiguous block of views: the split the multi-device projector
    # (ctlcu_group_project_volume) uses for a device list of `world` devices
    first = L.split_views(n_views, world)
    v0, v1 = first[rank], first[rank + 1]
    P = np.ascontiguousarray(P_all[v0:v1])
    mine = v1 - v0
    settings = Settings(accum={"fp64": L.ACCUM_FP64, "kahan": L.ACCUM_KAHAN, "fp32": L.ACCUM_FP32}[args.accum],
                        storage={"f32": L.F32, "bf16": L.BF16, "f16": L.F16}[args.storage],
                        interp_mode=L.INTERP_TEXTURE if args.interp == "texture" else L.INTERP_SOFTWARE,
                        kernel={"auto": L.KERNEL_AUTO, "gather": L.KERNEL_GATHER, "cells": L.KERNEL_CELLS,
                                 "pairs": L.KERNEL_PAIRS}[args.kernel],
                        block_rays=args.block_rays, views_per_block=args.views_per_block, lanes_x=args.lanes_x,
                        unroll=args.unroll)
    ctx = Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    vobj = VoxelVolume(vol, VOXEL)
    volume = ctx.volume(vobj, settings.storage)
    dP = torch.from_numpy(P).to(dev)
    out = torch.empty((mine, 1, ROWS, CHANNELS), dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    samples = ctx.count_samples(volume, P, CHANNELS, ROWS, settings)
    tuned = None
    if settings.kernel == L.KERNEL_AUTO and settings.interp_mode == L.INTERP_SOFTWARE:
        tuned = ctx.autotune(volume, P, CHANNELS, ROWS, settings)  # sample loop and launch shape for this job
    ran = ctx.tuned_settings(volume, 1, CHANNELS, ROWS, settings)  # what the timed calls run

    def step():
        ctx.project(volume, dP, CHANNELS, ROWS, settings, out=out, stream=ctx.stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        barrier(world)
        clocks = ClockSampler(local)
        clocks.start()
        l0 = ctx.launches()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        torch.cuda.synchronize()
        barrier(world)
        for i in range(args.steps):
            flush.zero_()  # L2 flush outside the timed events
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        launches = ctx.launches() - l0
        step_ms = [a.elapsed_time(b) for a, b in ev]
    own_ms = sum(step_ms)
    total_ms = max_over_ranks(own_ms, world)
    ms_per_step = total_ms / args.steps
    value = n_views * args.steps / (total_ms / 1e3)

    # Each step is one setup launch (about 5 us for 360 views) and one projection
    # launch, timed together by the events on their stream; the step time stands
    # for the projection kernel's launch time (the setup is < 0.01% of it).
    kernel_ms = own_ms / args.steps

    # e2e through the C ABI with host buffers (pinned): this rank's block
    h_vol = torch.from_numpy(vol).pin_memory()
    h_P = torch.from_numpy(P).pin_memory()
    h_out = torch.empty((mine, 1, ROWS, CHANNELS), dtype=torch.float32).pin_memory()
    desc_vol = VoxelVolume(h_vol.numpy(), VOXEL)
    # as many warm-up calls as device steps: with one, the first timed calls still ran
    # up to 8% slower and the end-to-end number varied from run to run
    for _ in range(max(1, args.warmup)):
        ctx.project_volume(desc_vol, h_P.numpy(), CHANNELS, ROWS, settings, out=h_out.numpy())
    barrier(world)
    e2e_ms = []
    for _ in range(max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.project_volume(desc_vol, h_P.numpy(), CHANNELS, ROWS, settings, out=h_out.numpy())
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    e2e_value = n_views * len(e2e_ms) / (e2e_total / 1e3)
    clk = clocks.stop()

    legs = None
    if world == 1 and not args.headline_only:
        legs = run_legs(args, ctx, vobj, volume, P, flush, stream, value)

    if rank == 0:
        b = 4 if settings.storage == L.F32 else 2
        alg_bytes = samples * 8 * b + 4 * mine * ROWS * CHANNELS
        props = torch.cuda.get_device_properties(dev)
        sms = props.multi_processor_count
        mhz = clk.get("sm_mhz") or 1965.0
        l1_peak = sms * 128 * mhz * 1e6 / 1e9  # GB/s
        achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
        loop = ran.kernel
        shape = ran.launch_shape()
        traffic = (CELLS_TRAFFIC_BYTES if loop == L.KERNEL_CELLS and mine == N_VIEWS and
                   settings.storage == L.F32 and settings.interp_mode == L.INTERP_SOFTWARE and
                   args.accum == CELLS_TRAFFIC_ACCUM and tuple(shape.values()) == CELLS_TRAFFIC_SHAPE else None)
        line = {
            "metric": METRIC, "value": value, "unit": "projections/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": {L.F32: "f32", L.BF16: "bf16", L.F16: "f16"}[settings.storage] + "-storage/f32-interp/"
                     + args.accum + "-accum",
            "data": "synthetic (seeded ellipsoid phantom, seeded jittered geometry)",
            "config": bench_config(world, n_views),
            "run": {"storage": {L.F32: "f32", L.BF16: "bf16", L.F16: "f16"}[settings.storage],
                    "accum": args.accum, "interp": args.interp, "kernel": args.kernel,
                    "loop": {L.KERNEL_CELLS: "cells", L.KERNEL_PAIRS: "pairs",
                             L.KERNEL_GATHER: "gather"}.get(loop, "auto"),
                    "launch_shape": shape, "views_of_rank0": [v0, v1]},
            "vs_baseline_note": "the reference publishes no number for this metric",
            "samples_per_step": samples,
            "gsamples_per_s": samples * args.steps / (own_ms / 1e3) / 1e9,
            "e2e": {"value": e2e_value, "unit": "projections/s",
                    "h2d_bytes_per_step": int(vol.nbytes + P.nbytes),
                    "d2h_bytes_per_step": int(h_out.numel() * 4),
                    "path": "ctlcu_project_volume, pinned host buffers (per rank: its block of views)"},
            "gpu_launches": int(launches),
            "autotune": None if tuned is None else {
                "chosen": {L.KERNEL_CELLS: "cells", L.KERNEL_PAIRS: "pairs", L.KERNEL_GATHER: "gather"}[tuned[0]],
                "ms_on_8_views": tuned[1]},
            "roofline": {"bound": "l1", "achieved": achieved, "peak": l1_peak, "unit": "GB/s",
                         "frac": achieved / l1_peak, "traffic": traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one full launch"
                                           if traffic else "not captured for this variant",
                         "peak_source": f"{sms} SMs x 128 B/clk x {mhz:.0f} MHz sampled SM clock",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         # the DRAM side: the captured traffic over this run's launch time, against
                         # the measured HBM copy rate (the bound that does not bind this kernel)
                         "dram_gb_s": traffic / (kernel_ms / 1e3) / 1e9 if traffic else None,
                         "dram_frac_of_hbm": traffic / (kernel_ms / 1e3) / 1e9 / hbm_peak() if traffic else None},
            "clocks": clk,
        }
        if legs is not None:
            line["legs"] = legs
        if world == 1 and not args.no_cpu_baseline:
            import oracle
            if oracle.ref_available():
                rate, n, dt = cpu_reference_rate(vol, P_all, args.cpu_seconds, os.cpu_count() or 1)
                line["cpu_baseline"] = {"value": rate, "unit": "projections/s", "cores": os.cpu_count(),
                                        "kind": "reference",
                                        "sample": f"{n} of {N_VIEWS} views evenly spaced, {dt:.1f} s"}
            # the FP64 formulation of the reference's CPU projector (RayCasterProjectorCPU,
            # raycasterprojectorcpu.cpp:132-285), as the oracle restates it, timed once beside it
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            oracle.project_fp64(vol, VOXEL, P_all[:1], CHANNELS, ROWS, threads=threads)
            t1 = time.perf_counter() - t0
            n = int(max(1, min(N_VIEWS, round(0.5 * args.cpu_seconds / max(t1, 1e-3)))))
            idx = np.linspace(0, N_VIEWS - 1, n).round().astype(int)
            t0 = time.perf_counter()
            oracle.project_fp64(vol, VOXEL, P_all[idx], CHANNELS, ROWS, threads=threads)
            dt = time.perf_counter() - t0
            line["cpu_fp64_twin"] = {"value": n / dt, "unit": "projections/s", "cores": threads, "kind": "port",
                                     "sample": f"{n} of {N_VIEWS} views evenly spaced, {dt:.1f} s"}
        print(json.dumps(line))
    volume.release()
    ctx.close()
    if _dist_on():
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_legs(args, ctx, vobj, volume, P, flush, stream, value_fp32):
    """The rest of the headline metric on one GPU: the FP64 accumulator, the
    plain FP32 gather loop, the batched BF16 form and DRR serving latency."""
    import torch

    from ctl_b200 import _lib as L
    from ctl_b200.projector import Settings
    V = P.shape[0]
    dP = torch.from_numpy(P).cuda()
    out = torch.empty((V, 1, ROWS, CHANNELS), dtype=torch.float32, device="cuda")
    steps = max(3, args.steps // 2)
    legs = {}

    def rate(ms):
        return V / (statistics.mean(ms) / 1e3)

    # the reference kernel's own accumulator type (FP64), same loop and shape
    s64 = Settings(accum=L.ACCUM_FP64)
    ms = _time_steps(lambda: ctx.project(volume, dP, CHANNELS, ROWS, s64, out=out, stream=ctx.stream), steps,
                     args.warmup, stream, flush.zero_)
    legs["accum_fp64"] = {"value": rate(ms), "unit": "projections/s", "ms_per_step": statistics.mean(ms),
                          "what": "FP32 storage, cell loop, FP64 accumulator"}
    # the plain FP32 CUDA projector: eight scalar loads per sample from the padded voxels
    sg = Settings(kernel=L.KERNEL_GATHER)
    ms = _time_steps(lambda: ctx.project(volume, dP, CHANNELS, ROWS, sg, out=out, stream=ctx.stream), steps,
                     args.warmup, stream, flush.zero_)
    plain = rate(ms)
    legs["plain_gather_fp32"] = {"value": plain, "unit": "projections/s", "ms_per_step": statistics.mean(ms),
                                 "what": "FP32 storage, gather loop (8 scalar loads per sample), Kahan accumulator"}
    # the batched BF16 form: BF16 storage, 8 requests of 45 views (clients of one volume)
    # in one CUDA graph replay (ctlcu_plan_launch), in the plan's faster form
    vb = ctx.volume(vobj, L.BF16)
    ctx.autotune(vb, P, CHANNELS, ROWS, Settings())
    parts = L.split_views(V, 8)
    reqs = [(vb, dP[parts[i]:parts[i + 1]], out[parts[i]:parts[i + 1]]) for i in range(8)]
    plan = ctx.plan(reqs, Settings())
    ms = _time_steps(lambda: plan.launch(ctx.stream), args.steps, args.warmup, stream, flush.zero_)
    batched = rate(ms)
    legs["batched_bf16"] = {"value": batched, "unit": "projections/s", "ms_per_step": statistics.mean(ms),
                            "what": "BF16 storage, 8 requests x 45 views, one CUDA graph replay per step "
                                    "(ctlcu_plan_launch)",
                            "plan": plan.info(),
                            "vs_plain_gather_fp32": batched / plain, "vs_drop_in_fp32": batched / value_fp32}
    plan.close()
    del reqs
    vb.release()
    torch.cuda.synchronize()
    legs["drr"] = drr_measurements(ctx, args, sweep=False)
    return legs


# ---- the other configurations (extra lines; the headline is the 256^3 -> 512^2 one above) ------

def _time_device(fn, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in ev:
        a.record(stream)
        fn()
        b.record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def _line(metric, value, unit, ms, args, config, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
         "vs_baseline": None, "data": "synthetic (seeded ellipsoid phantoms, seeded geometry)", "config": config}
    d.update(extra)
    print(json.dumps(d), flush=True)


def run_single_config(args, name):
    """c1 / c3: one volume, all views per step, resident; several sample-loop forms."""
    import torch

    from ctl_b200 import _lib as L
    from ctl_b200 import workloads as W
    from ctl_b200.projector import Context, Settings, VoxelVolume
    job = W.c1() if name == "c1" else W.c3()
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    V, M = job.pmats.shape[:2]
    dP = torch.from_numpy(job.pmats).cuda()
    out = torch.empty((V, M, job.rows, job.channels), device="cuda")
    forms = {"cells_fp64": Settings(accum=L.ACCUM_FP64), "cells_kahan": Settings(accum=L.ACCUM_KAHAN),
             "cells_fp32": Settings(accum=L.ACCUM_FP32),
             "gather_fp64": Settings(kernel=L.KERNEL_GATHER, accum=L.ACCUM_FP64),
             "texture_fp64": Settings(interp_mode=L.INTERP_TEXTURE, accum=L.ACCUM_FP64)}
    storages = {"f32": L.F32, "bf16": L.BF16}
    results, shapes = {}, {}
    for sname, storage in storages.items():
        vol = ctx.volume(VoxelVolume(job.volume, job.voxel), storage)
        for fname, s in forms.items():
            if storage == L.BF16 and fname == "texture_fp64":
                continue
            ms = _time_device(lambda: ctx.project(vol, dP, job.channels, job.rows, s, out=out, stream=ctx.stream),
                              args.steps, args.warmup, stream)
            results[f"{sname}_{fname}"] = V / (statistics.mean(ms) / 1e3)
        # the autotuned sample loop and launch shape (default settings: Kahan accumulation)
        ctx.autotune(vol, job.pmats, job.channels, job.rows)
        tuned = ctx.tuned_settings(vol, M, job.channels, job.rows)
        ms = _time_device(lambda: ctx.project(vol, dP, job.channels, job.rows, Settings(), out=out,
                                              stream=ctx.stream), args.steps, args.warmup, stream)
        results[f"{sname}_tuned_kahan"] = V / (statistics.mean(ms) / 1e3)
        shapes[sname] = dict(tuned.launch_shape(), loop={L.KERNEL_CELLS: "cells", L.KERNEL_PAIRS: "pairs",
                                                          L.KERNEL_GATHER: "gather"}[tuned.kernel])
        if sname == "f32":
            samples = ctx.count_samples(vol, job.pmats, job.channels, job.rows)
        vol.release()
    best = results["f32_tuned_kahan"]  # the automatic path once tuned
    ms = V / best * 1e3
    extra = {"forms_views_per_s": results, "tuned": shapes, "samples_per_step": samples,
             "gsamples_per_s": samples / (ms / 1e3) / 1e9}
    if name == "c3":
        # compulsory HBM traffic of one step: the FP32 volume read once and the
        # projections written once; beside it, the derived cell array (32 B per
        # cell, (n + 3) cells per axis) read once in place of the volume
        nz, ny, nx = (int(n) for n in job.volume.shape)
        out_bytes = V * M * job.rows * job.channels * 4
        vol_bytes = nx * ny * nz * 4
        cell_bytes = 32 * (nx + 3) * (ny + 3) * (nz + 3)
        t = ms / 1e3
        extra["hbm_compulsory"] = {
            "bytes_per_step": vol_bytes + out_bytes, "gb_s": (vol_bytes + out_bytes) / t / 1e9,
            "frac_of_hbm": (vol_bytes + out_bytes) / t / 1e9 / hbm_peak(), "hbm_peak_gb_s": hbm_peak(),
            "with_cell_array": {"bytes_per_step": cell_bytes + out_bytes, "gb_s": (cell_bytes + out_bytes) / t / 1e9,
                                "frac_of_hbm": (cell_bytes + out_bytes) / t / 1e9 / hbm_peak()}}
    if name == "c1" and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            vol_h = job.volume if isinstance(job.volume, np.ndarray) else job.volume.cpu().numpy()
            t0 = time.perf_counter()
            oracle.project_ref(vol_h, job.voxel, job.pmats, job.channels, job.rows, threads=os.cpu_count())
            dt = time.perf_counter() - t0
            extra["cpu_baseline"] = {"value": V / dt, "unit": "projections/s", "cores": os.cpu_count(),
                                     "kind": "reference", "sample": f"all {V} views, {dt:.1f} s"}
    _line(f"projections/s, {job.name}", best, "projections/s", ms, args,
          {"workload": job.name, "views_per_step": V, "modules": M}, **extra)
    ctx.close()


def run_geometry(args):
    """Projection matrices of the C3 acquisition (helical, 1440 views x 64 cylindrical
    modules of 16 x 16) encoded on the device, against the FP64 oracle port on one core."""
    import torch

    from ctl_b200 import encoder as E
    from ctl_b200.projector import Context
    n_views, modules = 1440, 64
    det = E.CylindricalDetector((16, 16), (1.0, 1.0), modules, 16.0 / 1040.0, 0.0)
    setup = E.AcquisitionSetup(det, E.TubularGantry(1040.0, 570.0), n_views)
    setup.apply_preparation_protocol(E.HelicalTrajectory(math.radians(1.0), 256.0 / n_views, -128.0))
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = torch.empty((n_views, modules, 3, 4), dtype=torch.float64, device="cuda")
    ms = _time_device(lambda: E.GeometryEncoder.encode_full_geometry(setup, ctx, out=out, stream=ctx.stream),
                      args.steps, args.warmup, stream)
    n = n_views * modules
    t_ms = statistics.mean(ms)
    host = np.empty((n_views, modules, 3, 4))
    e2e = []
    for _ in range(max(1, args.e2e_steps)):
        t0 = time.perf_counter()
        E.GeometryEncoder.encode_full_geometry(setup, ctx, out=host)
        e2e.append(time.perf_counter() - t0)
    extra = {"e2e": {"value": n / statistics.mean(e2e), "unit": "matrices/s", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": int(host.nbytes), "path": "ctlcu_encode_geometry into host memory"},
             "gpu_launches": 1,
             "roofline": {"bound": "launch", "achieved": host.nbytes / (t_ms / 1e3) / 1e9, "unit": "GB/s",
                          "note": "one launch of 92160 threads writing 96 B each: latency-bound, "
                                  "far below the HBM ceiling by construction"}}
    if not args.no_cpu_baseline:
        from oracle import geometry_oracle as GO
        d = GO.Detector(16, 16, 1.0, 1.0, modules=modules, angulation=16.0 / 1040.0, spacing=0.0)
        t = GO.Trajectory("helical", sdd=1040.0, sid=570.0, angle_increment=math.radians(1.0),
                          pitch_increment=256.0 / n_views, start_pitch=-128.0)
        sample = 48
        t0 = time.perf_counter()
        GO.encode_full_geometry(d, t, sample)
        dt = time.perf_counter() - t0
        extra["cpu_baseline"] = {"value": sample * modules / dt, "unit": "matrices/s", "cores": 1, "kind": "port",
                                 "sample": f"first {sample} of {n_views} views x {modules} modules, {dt:.2f} s"}
    _line("projection matrices/s, helical 1440 views x 64 cylindrical modules (GeometryEncoder)",
          n / (t_ms / 1e3), "matrices/s", t_ms, args,
          {"workload": "CylindricalDetector(16x16 px, 64 modules) on TubularGantry(1040, 570), "
                       "HelicalTrajectory(1 deg, 256/1440 mm, start -128 mm), 1440 views"}, **extra)
    ctx.close()


def run_postops(args):
    """Poisson noise (PoissonNoiseExtension) on the 256^3 -> 360 x 512^2 projections, on
    the device, against the reference's own noise engine (per-view std::mt19937_64 with
    libstdc++'s distributions, oracle/poisson_ref.cpp) on the host."""
    import torch

    from ctl_b200.projector import Context, Settings, VoxelVolume
    n_views = args.views
    vol, P = make_inputs(n_views)
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    volume = ctx.volume(VoxelVolume(vol, VOXEL))
    dP = torch.from_numpy(P).cuda()
    clean = ctx.project(volume, dP, CHANNELS, ROWS, Settings(), stream=ctx.stream)
    torch.cuda.synchronize()
    i0 = np.array([1.0e4], np.float32)   # photons per pixel: counts from 1e4 down to single digits
    work = torch.empty_like(clean)
    times = []
    with torch.cuda.stream(stream):
        for i in range(args.warmup + args.steps):
            work.copy_(clean)   # fresh input each step, outside the events (the noise is in place)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.poisson_noise(work, i0, SEED_NOISE + i, stream=ctx.stream)
            b.record(stream)
            torch.cuda.synchronize()
            if i >= args.warmup:
                times.append(a.elapsed_time(b))
    n = clean.numel()
    t_ms = statistics.mean(times)
    host = clean.cpu().numpy()
    e2e = []
    for i in range(max(1, args.e2e_steps)):
        h = host.copy()
        t0 = time.perf_counter()
        ctx.poisson_noise(h, i0, SEED_NOISE + i)
        e2e.append(time.perf_counter() - t0)
    extra = {"e2e": {"value": n_views / statistics.mean(e2e), "unit": "projections/s",
                     "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(host.nbytes),
                     "path": "ctlcu_poisson_noise on host data"},
             "gpu_launches": 1,
             "pixels_per_step": int(n),
             "roofline": {"bound": "hbm", "achieved": 8.0 * n / (t_ms / 1e3) / 1e9, "peak": hbm_peak(),
                          "unit": "GB/s", "frac": 8.0 * n / (t_ms / 1e3) / 1e9 / hbm_peak(),
                          "algorithmic_bytes_per_launch": int(8 * n),
                          "note": "4 B read + 4 B write per pixel; the FP64 sampler (PTRS with lgamma) "
                                  "is the actual limit, not HBM"}}
    if not args.no_cpu_baseline:
        import oracle
        sample = 4
        x = host[:sample].copy()
        t0 = time.perf_counter()
        oracle.poisson_noise_reference(x, i0, SEED_NOISE)
        dt = time.perf_counter() - t0
        extra["cpu_baseline"] = {"value": sample / dt, "unit": "projections/s", "cores": 1, "kind": "port",
                                 "sample": f"{sample} of {n_views} views with the reference's per-view "
                                           f"mt19937_64 + std:: distributions, {dt:.2f} s"}
    _line(f"projections/s through Poisson noise (PoissonNoiseExtension), {n_views} x 512^2, i0 = 1e4",
          n_views / (t_ms / 1e3), "projections/s", t_ms, args,
          {"workload": WORKLOAD + "; then Poisson noise, i0 = 1e4 photons/pixel"}, **extra)
    volume.release()
    ctx.close()


def run_den(args):
    """The 360 x 512^2 projections written to a DEN file straight from device memory
    (ctlcu_den_write: pinned double-buffered staging, copies overlapping the writes),
    against CTL's path: every view copied to a host ProjectionData, then written."""
    import shutil
    import tempfile

    import torch

    from ctl_b200 import den as D
    from ctl_b200.projector import Context
    ctx = Context(0)
    rng = np.random.default_rng(5)
    dev = torch.from_numpy(rng.random((N_VIEWS, 1, ROWS, CHANNELS), dtype=np.float32)).cuda()
    nbytes = dev.numel() * 4
    tmp = tempfile.mkdtemp(prefix="den_bench_")
    try:
        path = os.path.join(tmp, "proj.den")
        times = []
        for i in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            D.save_projections(ctx, dev, path)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
        # CTL's order of work: per-view device->host copies into host memory, then the file
        ref = []
        host = np.empty((N_VIEWS, 1, ROWS, CHANNELS), np.float32)
        for i in range(max(1, min(3, args.steps))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for v in range(N_VIEWS):
                host[v] = dev[v].cpu().numpy()
            D.write_den(os.path.join(tmp, "ref.den"), host.reshape(N_VIEWS, ROWS, CHANNELS))
            ref.append(time.perf_counter() - t0)
        t = statistics.mean(times)
        # the same two paths into /dev/null: the copy pipeline without the file system
        null = []
        for i in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            D.save_projections(ctx, dev, "/dev/null")
            null.append(time.perf_counter() - t0)
        null_ref = []
        for i in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for v in range(N_VIEWS):
                host[v] = dev[v].cpu().numpy()
            D.write_den("/dev/null", host.reshape(N_VIEWS, ROWS, CHANNELS))
            null_ref.append(time.perf_counter() - t0)
        extra = {"e2e": {"value": nbytes / t / 1e9, "unit": "GB/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": int(nbytes), "path": "ctlcu_den_write from device memory"},
                 "gpu_launches": 0,
                 "per_view_copy_then_write_gb_s": nbytes / statistics.mean(ref) / 1e9,
                 "to_dev_null_gb_s": nbytes / min(null) / 1e9,
                 "per_view_copy_then_write_to_dev_null_gb_s": nbytes / min(null_ref) / 1e9,
                 "target": f"{tmp} (page cache; no fsync)",
                 "roofline": {"bound": "pcie/host", "achieved": nbytes / t / 1e9, "unit": "GB/s",
                              "note": "device-to-host copies and file writes, overlapped; no kernel"}}
        _line("GB/s writing 360 x 512^2 float32 projections to a DEN file from device memory",
              nbytes / t / 1e9, "GB/s", t * 1e3, args,
              {"workload": "360 x 512 x 512 float32 projections (377 MB) -> DEN file"}, **extra)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        ctx.close()


def run_focalspot(args):
    """ArealFocalSpotExtension with 3 x 3 focal-spot samples (1 x 1 mm spot) over the
    256^3 phantom and a 360-view C-arm short scan onto a 512^2 flat panel (0.6 mm):
    geometry, projection and intensity averaging as one batched pass each, against the
    reference's call pattern (one nested project() per sample, volume re-uploaded, host
    averaging) on this library, and the reference kernel on the host cores."""
    import torch

    from ctl_b200 import encoder as E
    from ctl_b200.extensions import ArealFocalSpotExtension
    from ctl_b200.projector import Context, Settings, VoxelVolume
    from ctl_b200 import phantom as Ph
    vol = Ph.ellipsoid_phantom(SHAPE, VOXEL, 40, seed=2)
    ctx = Context(0)
    setup = E.AcquisitionSetup(E.FlatPanelDetector((CHANNELS, ROWS), (0.6, 0.6)), E.CarmGantry(1200.0), N_VIEWS)
    setup.apply_preparation_protocol(E.ShortScanTrajectory(750.0, 0.0, math.radians(200.0)))
    ext = ArealFocalSpotExtension(ctx, discretization=(3, 3))
    ext.configure(setup, (1.0, 1.0))
    resident = ctx.volume(VoxelVolume(vol, VOXEL))
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        ext.project(resident)

    times = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        step()
        b.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(a.elapsed_time(b))
    t_ms = statistics.mean(times)
    # end to end from a host volume to a host result
    vobj = VoxelVolume(vol, VOXEL)
    e2e = []
    for _ in range(max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ext2 = ArealFocalSpotExtension(ctx, discretization=(3, 3))
        ext2.configure(setup, (1.0, 1.0))
        ext2.project(vobj).cpu()
        e2e.append(time.perf_counter() - t0)
        ext2.release()
    # the reference's call pattern on this library: per sample, configure + project_volume
    shifts = ext.source_shifts()
    pattern = []
    for _ in range(2):
        t0 = time.perf_counter()
        acc = None
        for s in shifts:
            P = E.GeometryEncoder.encode_full_geometry(setup, ctx, source_shifts=s[None])
            p = ctx.project_volume(vobj, P, CHANNELS, ROWS, Settings())
            acc = np.exp(-p) if acc is None else acc + np.exp(-p)
        np.log(len(shifts) / acc)
        pattern.append(time.perf_counter() - t0)
    extra = {"e2e": {"value": N_VIEWS / statistics.mean(e2e), "unit": "projections/s",
                     "h2d_bytes_per_step": int(vol.nbytes), "d2h_bytes_per_step": int(N_VIEWS * ROWS * CHANNELS * 4),
                     "path": "ArealFocalSpotExtension.project(VoxelVolume) -> host"},
             "gpu_launches": 4,   # geometry, ray setup, projection, averaging
             "samples": 9,
             "reference_call_pattern_views_s": N_VIEWS / min(pattern)}
    if not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            P = E.GeometryEncoder.encode_full_geometry(setup, ctx, source_shifts=shifts)
            pick = P[[0, 180, 4 * N_VIEWS + 90]]   # three sample-views spread over the scan
            t0 = time.perf_counter()
            oracle.project_ref(vol, VOXEL, pick, CHANNELS, ROWS, threads=os.cpu_count())
            dt = time.perf_counter() - t0
            extra["cpu_baseline"] = {"value": len(pick) / dt / 9.0, "unit": "projections/s",
                                     "cores": os.cpu_count(), "kind": "reference",
                                     "sample": f"{len(pick)} sample-views of the reference kernel, {dt:.1f} s; "
                                               "9 sample-views per output view"}
    _line("projections/s through ArealFocalSpotExtension (3 x 3 samples), 256^3 -> 360 x 512^2",
          N_VIEWS / (t_ms / 1e3), "projections/s", t_ms, args,
          {"workload": "256^3 phantom, C-arm short scan 200 deg, 360 views, 512^2 @ 0.6 mm, "
                       "focal spot 1 x 1 mm sampled 3 x 3 (3240 sample-views per step)"}, **extra)
    resident.release()
    ext.release()
    ctx.close()


def run_spectral(args):
    """SpectralEffectsExtension around projector | PoissonNoiseExtension: two material
    densities (256^3 water and bone phantoms) onto the 360-view 512^2 scan, 30 energy bins,
    10^5 photons per pixel spread over the bins.  Ours: one batched projection of the two
    densities, then all 60 (bin, material) noise draws and the bin combine in one kernel.
    The reference makes 60 projections (each with its volume upload) and 60 noise passes."""
    import torch

    from ctl_b200 import phantom as Ph
    from ctl_b200.extensions import SpectralEffectsExtension
    from ctl_b200.projector import Context, Settings, VoxelVolume
    n_bins = 30
    water = Ph.ellipsoid_phantom(SHAPE, VOXEL, 40, seed=2) * 50.0   # density-like values
    bone = Ph.ellipsoid_phantom(SHAPE, VOXEL, 8, seed=3) * 10.0
    n_views = args.views
    _, P = make_inputs(n_views)
    e = np.linspace(20.0, 120.0, n_bins)                            # keV
    spectrum = np.exp(-0.5 * ((e - 60.0) / 20.0) ** 2)
    spectrum /= spectrum.sum()
    mu = np.stack([0.02 * (30.0 / e) ** 1.5 + 0.015, 0.05 * (30.0 / e) ** 2.5 + 0.02], axis=1).astype(np.float32)
    inten = np.repeat((spectrum * 1e5)[:, None], n_views, axis=1)   # [bins][views]
    total = inten.sum(0)
    i0 = (spectrum * 1e5)[:, None].astype(np.float32)              # [bins][modules]
    ctx = Context(0)
    ext = SpectralEffectsExtension(ctx)
    ext.configure(P, CHANNELS, ROWS, mu, inten, total, None, photons_per_pixel=i0, fixed_seed=SEED_NOISE)
    vols = [VoxelVolume(water, VOXEL), VoxelVolume(bone, VOXEL)]
    # the two density projections alone, resident, for the split of the step
    res = [ctx.volume(v) for v in vols]
    dP = torch.from_numpy(P).cuda()
    projs = torch.empty((2, n_views, 1, ROWS, CHANNELS), device="cuda")

    def timed(fn):
        out = []
        for i in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                out.append(a.elapsed_time(b))
        return statistics.mean(out)

    t_step = timed(lambda: ext.project(vols))
    t_proj = timed(lambda: (ctx.project_batch([(r, dP, projs[m]) for m, r in enumerate(res)], Settings()),
                            ctx.sync()))
    calls = ext.nested_calls()
    # the material volumes stay resident in the extension after the first (warm-up) call, so a
    # step is the batched projection (setup + persistent kernel) and the noise-and-combine kernel
    extra = {"split_ms": {"material_projections": t_proj, "noise_draws_and_combine": t_step - t_proj},
             "nested_calls_per_step": calls, "gpu_launches": 3}
    if not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            pick = P[[0, n_views // 2]]
            t0 = time.perf_counter()
            oracle.project_ref(water, VOXEL, pick, CHANNELS, ROWS, threads=os.cpu_count())
            dt = time.perf_counter() - t0
            extra["cpu_baseline"] = {"value": len(pick) / dt / calls, "unit": "projections/s",
                                     "cores": os.cpu_count(), "kind": "reference",
                                     "sample": f"{len(pick)} views of the reference kernel, {dt:.1f} s; "
                                               f"{calls} projections per output view (noise passes not counted)"}
    _line("projections/s through SpectralEffectsExtension + Poisson noise (30 bins, 2 materials), "
          f"256^3 -> {n_views} x 512^2", n_views / (t_step / 1e3), "projections/s", t_step, args,
          {"workload": "water + bone density phantoms 256^3, short scan 360 x 512^2, 30 bins, "
                       "1e5 photons per pixel, projector | PoissonNoiseExtension nested"}, **extra)
    for r in res:
        r.release()
    ctx.close()


def hbm_peak() -> float:
    """The measured HBM copy bandwidth of this pool's B200s (GB/s), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


SEED_NOISE = 20240611


def run_c4(args):
    """64 uneven volumes: one plan (a CUDA graph replay) vs 64 sequential calls."""
    import torch

    from ctl_b200 import _lib as L
    from ctl_b200 import workloads as W
    from ctl_b200.projector import Context, Settings, VoxelVolume
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    jobs = W.c4(n_volumes=args.volumes)
    total_views = sum(j.pmats.shape[0] for j in jobs)
    for storage_name, storage in (("f32", L.F32), ("bf16", L.BF16)):
        vols = [ctx.volume(VoxelVolume(j.volume, j.voxel), storage) for j in jobs]
        reqs = []
        for j, v in zip(jobs, vols):
            V, M = j.pmats.shape[:2]
            reqs.append((v, torch.from_numpy(j.pmats).cuda(), torch.empty((V, M, j.rows, j.channels), device="cuda")))
        plan = ctx.plan(reqs, Settings())
        ms_plan = _time_device(lambda: plan.launch(ctx.stream), args.steps, args.warmup, stream)

        def sequential(kernel):
            s = Settings(kernel=kernel)
            for (v, P, out), j in zip(reqs, jobs):
                ctx.project(v, P, j.channels, j.rows, s, out=out, stream=ctx.stream)
        ms_seq = _time_device(lambda: sequential(L.KERNEL_CELLS), max(2, args.steps // 3), 1, stream)
        ms_plain = _time_device(lambda: sequential(L.KERNEL_GATHER), max(2, args.steps // 3), 1, stream)
        info = plan.info()
        plan.close()
        v_plan = total_views / (statistics.mean(ms_plan) / 1e3)
        _line(f"projections/s, 64 uneven volumes batched ({storage_name} storage)", v_plan, "projections/s",
              statistics.mean(ms_plan), args,
              {"workload": "64 volumes (edges 96-256), 30-360 views each, detectors 256^2-768x512",
               "views_per_step": total_views, "storage": storage_name},
              plan=info, sequential_cells_views_per_s=total_views / (statistics.mean(ms_seq) / 1e3),
              sequential_plain_gather_views_per_s=total_views / (statistics.mean(ms_plain) / 1e3))
        for v in vols:
            v.release()
        del reqs
        torch.cuda.empty_cache()
    ctx.close()


def drr_measurements(ctx, args, sweep: bool = True) -> dict:
    """DRR serving on 8 resident 256^3 BF16 volumes: capacity, latency at 2000
    requests/s offered, the highest offered rate whose p99 stays under 5 ms, and
    the sample count the 2000/s stream asks for."""
    from ctl_b200 import _lib as L
    from ctl_b200 import workloads as W
    from ctl_b200.projector import Settings, VoxelVolume
    from ctl_b200.serving import DRRServer, poisson_requests
    vols = [ctx.volume(VoxelVolume(v, (1.0, 1.0, 1.0)), L.BF16) for v in W.c5_volumes()]
    kernel = {"auto": L.KERNEL_AUTO, "gather": L.KERNEL_GATHER, "cells": L.KERNEL_CELLS,
              "pairs": L.KERNEL_PAIRS}[args.kernel]
    settings = Settings(kernel=kernel)
    # 4 streams and batches of at most 12 views: a batch's launches hold the SMs until
    # they are done, so bounding its views bounds how long later requests wait behind it
    # (a sweep of 1-4 streams and 12-32 views gave this the highest capacity and the
    # lowest p99 at 700-900 requests/s).  24 GB of the 40 GB budget are reserved for
    # results up front (the volumes and their cells take 4.7 GB): no batch waits for the
    # allocator to grow
    server = DRRServer(ctx, vols, 256, 256, settings, streams=4, max_batch=256,
                       budget_bytes=40 * 10**9, max_batch_views=12, reserve_bytes=24 * 10**9)
    base = W.c5_base_view()
    server.warm_up(typical_pmats=np.repeat(base[None], 8, axis=0) if kernel == L.KERNEL_AUTO else None)
    # capacity: all requests offered at once.  The first run of this size also grows the
    # device allocators and ran up to 30% slower, so one untimed run comes first
    server.run(poisson_requests(1e7, 2000, len(vols), base, seed=49))
    n_cap = 3 if sweep else 1
    caps = [server.run(poisson_requests(1e7, 2000, len(vols), base, seed=50 + 100 * i)).summary()
            for i in range(n_cap)]
    caps.sort(key=lambda c: c["throughput_req_s"])
    cap = dict(caps[len(caps) // 2], runs_req_s=[c["throughput_req_s"] for c in caps])
    rate = 2000.0
    stream_2000 = poisson_requests(rate, int(rate * args.serve_seconds), len(vols), base, seed=51)
    at = server.run(stream_2000).summary()
    # the work the 2000/s stream asks for: exact reference-scheme samples of its requests
    samples = 0
    for k, v in enumerate(vols):
        mats = [r.pmats for r in stream_2000 if r.volume == k]
        if mats:
            samples += ctx.count_samples(v, np.concatenate(mats), 256, 256, settings)
    n_req = len(stream_2000)
    n_views = sum(int(r.pmats.shape[0]) for r in stream_2000)
    span_s = n_req / rate
    # offered-rate sweep: the highest rate whose p99 stays under 5 ms
    fracs = (0.2, 0.35, 0.5, 0.65, 0.75, 0.85) if sweep else (0.35, 0.5, 0.65, 0.75)
    points = []
    for frac in fracs:
        r_off = frac * cap["throughput_req_s"]
        sm = server.run(poisson_requests(r_off, max(200, int(r_off * args.serve_seconds)), len(vols), base,
                                         seed=52 + int(100 * frac))).summary()
        points.append(dict(sm, offered_req_s=r_off))
    ok = [q["offered_req_s"] for q in points if q["p99_ms"] < 5.0]
    res = {"unit": "ms", "offered_req_s": rate, "p50_ms": at["p50_ms"], "p95_ms": at["p95_ms"],
           "p99_ms": at["p99_ms"], "achieved_req_s": at["throughput_req_s"],
           "mean_requests_per_batch": at["mean_requests_per_batch"], "at_2000": at, "capacity": cap,
           "sweep": points, "max_rate_p99_under_5ms": max(ok) if ok else None,
           "work_at_2000": {"requests": n_req, "views": n_views, "samples": samples,
                            "samples_per_view": samples / max(n_views, 1),
                            "samples_per_s_needed": samples / span_s,
                            "samples_per_s_at_capacity": samples / n_views * cap["throughput_views_s"]},
           "workload": "8 resident 256^3 BF16 volumes; Poisson 2000/s; 1-16 perturbed views of 256^2 @1.2 mm; "
                       "40 GB budget (24 GB reserved for results); 4 streams, <= 12 views per batch",
           "launch_shapes": [ctx.tuned_settings(v, 1, 256, 256, settings).launch_shape() for v in vols]}
    for v in vols:
        v.release()
    return res


def run_c5(args):
    """DRR serving: capacity, then latency percentiles at 2000 requests/s offered."""
    from ctl_b200.projector import Context
    ctx = Context(0)
    d = drr_measurements(ctx, args, sweep=True)
    _line("p99 DRR latency at 2000 requests/s (8 x 256^3 BF16, 1-16 views of 256^2)", d["p99_ms"], "ms",
          d["p50_ms"], args, {"workload": d["workload"], "budget_bytes": 40 * 10**9}, higher_is_better=False,
          serving=d)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--accum", choices=["fp64", "kahan", "fp32"], default="kahan")
    ap.add_argument("--storage", choices=["f32", "bf16", "f16"], default="f32")
    ap.add_argument("--interp", choices=["software", "texture"], default="software")
    ap.add_argument("--kernel", choices=["auto", "gather", "cells", "pairs"], default="auto")
    # launch shape (0 = autotuned with --kernel auto, else the library default)
    ap.add_argument("--block-rays", type=int, default=0, choices=[0, 128, 256, 512])
    ap.add_argument("--views-per-block", type=int, default=0, choices=[0, 1, 2, 4])
    ap.add_argument("--lanes-x", type=int, default=0, choices=[0, 4, 8])
    ap.add_argument("--unroll", type=int, default=0, choices=[0, 2, 4, 8])
    ap.add_argument("--views", type=int, default=N_VIEWS,
                    help="views per step (360 = the configuration; fewer = a small profiling case)")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-views", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", choices=["c1", "c2", "c3", "c4", "c5", "geometry", "postops", "den", "focalspot",
                                         "spectral"],
                    default="c2",
                    help="c2 (default) is the headline; the others print extra lines")
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--volumes", type=int, default=64,
                    help="c4: the first N of the 64 uneven volumes (fewer = a small profiling case)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the one-GPU legs (FP64 accumulator, gather, batched BF16, DRR serving)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config in ("c1", "c3"):
        return run_single_config(args, args.config)
    if args.config == "c4":
        return run_c4(args)
    if args.config == "c5":
        return run_c5(args)
    if args.config == "geometry":
        return run_geometry(args)
    if args.config == "postops":
        return run_postops(args)
    if args.config == "den":
        return run_den(args)
    if args.config == "focalspot":
        return run_focalspot(args)
    if args.config == "spectral":
        return run_spectral(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
