#!/usr/bin/env python
"""Benchmark of the RSFE Split-Bregman segmentation path on B200.

Metric: Gvoxel-iterations/s = voxels x outer iterations / seconds, whole job.
Workload (one step): one segmentation of a 256^3 FP32 volume (8 ellipsoids,
semi-axes 10-40, intensities 0.6-0.9, bias ramp 0.7->1.3 along z, noise 0.05,
seeded synthetic data), sigma 3, lamda1 = lamda2 = 1, epsilon 1e-3, lamda 0.5,
Dirichlet boundary, 100 outer iterations, each solving the Poisson step with
red-black Gauss-Seidel to relative residual 1e-6. The working set (~2 GB) is far
above the 126 MB L2, so no flush is needed between steps.

Arms:
  default            the sm_100a library through its C ABI (one rank per GPU under
                     torchrun; each rank segments its own volume: weak scaling)
  --impl reference   the reference's own C++ code (oracle/_ref, compiled from the
                     reference headers with headless shims) on the host cores, one
                     outer iteration of the same 256^3 workload per step, rank 0 only

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import csv
import importlib
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RSFE-SB Gvoxel-iters/s @256^3 (FP32, RB Gauss-Seidel to rel. residual 1e-6)"
UNIT = "Gvoxel-iters/s"
SHAPE = (256, 256, 256)
MAXITER = 100
PARAMS = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, epsilon=1e-3, lamda=0.5, dt=1.0, a0=0.0,
              b0=1.0, bc=2, maxiter=MAXITER, tol=0.0, gs_rel_res_tol=1e-6, gs_check_every=0,
              gs_max_sweeps=1000, omega=1.0)

# Algorithmic bytes per voxel of one launch of each loop kernel (FP32): the
# compulsory reads and writes of the fields it consumes and produces.
ALGO_BYTES_PER_VOXEL = {
    "rb_half": 6.0,           # other colour read 2, own b_eff read 2, own colour write 2
    "rb_residual": 8.0,       # u read 4, b_eff read 4
    "conv_k_heaviside": 24.0,  # phi, u0 read 8; four stage-1 fields write 16
    "conv_s_j4": 32.0,        # four fields read 16, write 16
    "conv_i_fit": 24.0,       # four fields read 16; the pair (l1 f1 - l2 f2, ...) write 8
    "conv_s_j2": 16.0,        # pair read 8, write 8
    "conv_k_rhs": 28.0,       # pair 8, u0 4, div(d-b) 4, phi 4 read; packed b_eff 4, u 4 write
    "div": 16.0,              # d-b read 12, div write 4
    "clamp_tol": 12.0,        # packed u read 4, phiold read 4, phi write 4
    "bregman": 44.0,          # phi 4, b 12, g 4 read; b 12, d-b 12 write
}

WORKLOADS = {
    # the 256^3 workload (the headline)
    "c2": dict(shape=(256, 256, 256), maxiter=100, sigma=3.0),
    # the 512x512x320 CT-shaped single volume
    "c3": dict(shape=(512, 512, 320), maxiter=200, sigma=4.0),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except Exception as e:  # nvidia-smi missing: report no clocks
            log("clock sampler unavailable:", e)
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for r in csv.reader(open(self.path)):
            if len(r) < 9:
                continue
            try:
                rows.append([x.strip() for x in r])
            except Exception:
                pass
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# --------------------------------------------------------------------- GPU arm
def unet_flop_estimate(shape):
    """FLOPs (2 per multiply-add) of one inference of the learned warm start's network:
    3 levels of two 3x3x3 convolutions (16, 32, 64 channels; 4 input fields: rhs,
    previous u, div(d - b), phi), 2x down- and up-sampling, skip connections
    concatenated, a 1x1x1 output convolution."""
    n1 = shape[0] * shape[1] * shape[2]
    n2, n3 = n1 / 8.0, n1 / 64.0
    k = 27
    macs = n1 * k * (4 * 16 + 16 * 16)            # level 1, encoder
    macs += n2 * k * (16 * 32 + 32 * 32)          # level 2, encoder
    macs += n3 * k * (32 * 64 + 64 * 64)          # level 3
    macs += n3 * 8 * 64 * 32 + n2 * 8 * 32 * 16   # 2x2x2 transposed convolutions
    macs += n2 * k * (64 * 32 + 32 * 32)          # level 2, decoder (skip concatenated)
    macs += n1 * k * (32 * 16 + 16 * 16)          # level 1, decoder
    macs += n1 * 16                               # output
    return 2.0 * macs


def bf16_peak_tflops():
    """Dense bf16 peak (burst) in TFLOP/s and where it comes from."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def unet_forward_ms(shape, dev, reps=5):
    """Device time of one inference of the same network (layers as in
    unet_flop_estimate, ReLU after each 3x3x3 convolution, 2x max-pooling down,
    2x2x2 transposed convolutions up) run by the cuDNN convolutions behind torch.nn:
    bf16 weights and activations, channels-last, random weights. A library network,
    timed only to bound what a learned warm start could gain; it is not on the path."""
    import torch
    import torch.nn as nn

    class Block(nn.Sequential):
        def __init__(self, cin, cout):
            super().__init__(nn.Conv3d(cin, cout, 3, padding=1), nn.ReLU(inplace=True),
                             nn.Conv3d(cout, cout, 3, padding=1), nn.ReLU(inplace=True))

    class UNet(nn.Module):
        def __init__(self):
            super().__init__()
            self.e1, self.e2, self.e3 = Block(4, 16), Block(16, 32), Block(32, 64)
            self.up2, self.up1 = nn.ConvTranspose3d(64, 32, 2, 2), nn.ConvTranspose3d(32, 16, 2, 2)
            self.d2, self.d1 = Block(64, 32), Block(32, 16)
            self.out = nn.Conv3d(16, 1, 1)

        def forward(self, x):
            a = self.e1(x)
            b = self.e2(nn.functional.max_pool3d(a, 2))
            c = self.e3(nn.functional.max_pool3d(b, 2))
            b = self.d2(torch.cat([self.up2(c), b], 1))
            return self.out(self.d1(torch.cat([self.up1(b), a], 1)))

    prev = torch.backends.cudnn.benchmark
    torch.backends.cudnn.benchmark = True
    try:
        net = UNet().to(dev, torch.bfloat16).to(memory_format=torch.channels_last_3d).eval()
        x = torch.randn((1, 4) + tuple(shape), device=dev, dtype=torch.bfloat16)
        x = x.contiguous(memory_format=torch.channels_last_3d)
        with torch.inference_mode():
            for _ in range(3):
                net(x)
            ts = []
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                net(x)
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
        del net, x
        torch.cuda.empty_cache()
        return sorted(ts)[len(ts) // 2]
    finally:
        torch.backends.cudnn.benchmark = prev


def learned_warm_start(pkg, ctx, shape, dev, stream, unet_flop, bf16_peak):
    """The learned warm start measured: the project's own network (tcgen05 kernels) on
    one 256^3 inference, and time-to-tolerance learned against plain on held-out
    volumes (two-ellipsoid generator, seeds 1000 and 1001), with the weights trained
    by `python -m 3dimagetoolkit_b200.warmstart train` (128^3, seeds 0-199)."""
    import torch

    ws = importlib.import_module("3dimagetoolkit_b200.warmstart")
    out = {}
    if not os.path.exists(ws.WEIGHTS):
        return {"measured": None, "why": "no trained weights at " + os.path.relpath(ws.WEIGHTS, ROOT)}
    try:
        with pkg.UNet(ctx, seed=0) as net:
            meta = ws.load(net)
            out["training"] = {k: (v.tolist() if v.size > 1 else v.item()) for k, v in meta.items()
                               if k != "losses"}
            with torch.cuda.stream(stream):
                x = torch.randn((1, 4) + tuple(shape), device=dev, dtype=torch.float32)
                for _ in range(2):
                    net.forward(x)
                ts = []
                for _ in range(5):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    net.forward(x)
                    e1.record(stream)
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
            own_ms = sorted(ts)[len(ts) // 2]
            out["unet_ms_own_tcgen05"] = own_ms
            out["unet_own_tflops"] = unet_flop / (own_ms * 1e-3) / 1e12
            out["unet_own_frac_of_bf16_peak"] = out["unet_own_tflops"] / bf16_peak
            ev = ws.evaluate(ctx, net, [1000, 1001], shape=tuple(shape))
            out["measured"] = ev["mean"]
            out["per_volume"] = ev["per_volume"]
    except Exception as exc:  # reported, the rest of the line stands
        out["measured"] = None
        out["error"] = f"{type(exc).__name__}: {exc}"[:300]
    return out


def half_sweep_us(ctx, shape, dev, stream):
    """Device time of one red-black half-sweep inside a Poisson solve, in us."""
    import torch

    with torch.cuda.stream(stream):  # every tensor op ordered with the library's launches
        g = torch.Generator(device=dev)
        g.manual_seed(11)
        u = torch.rand(shape, device=dev, dtype=torch.float32, generator=g)
        b = torch.rand(shape, device=dev, dtype=torch.float32, generator=g) - 0.5

        def solve_ms(sweeps):
            uu = u.clone()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.poisson_solve(uu, b, bc_type=2, tol=0.0, max_sweeps=sweeps, check_every=sweeps)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)

        solve_ms(2)
        solve_ms(202)
        d = sorted(solve_ms(202) - solve_ms(2) for _ in range(3))
    return d[1] * 1000.0 / 400.0


def run_gpu(args):
    import numpy as np
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    pkg = importlib.import_module("3dimagetoolkit_b200")

    wl = WORKLOADS[args.workload]
    if args.size:
        dims = [int(v) for v in args.size.split(",")]
        shape = tuple(dims) if len(dims) == 3 else (dims[0],) * 3
    else:
        shape = wl["shape"]
    n = shape[0] * shape[1] * shape[2]
    if args.workload == "c3" and not args.size:
        u0_np, phi0_np = pkg.synth.config_volume("c3", seed=args.seed + rank, dtype=np.float32)
    elif args.size:
        u0_np = pkg.synth.ellipsoids(shape, args.seed + rank, n=8, semi_axes=(10, 40),
                                     fg_range=(0.6, 0.9), bias=(0.7, 1.3), noise=0.05,
                                     dtype=np.float32)
        phi0_np = pkg.synth.sphere_phi0(shape, 20.0, dtype=np.float32)
    else:
        u0_np, phi0_np = pkg.synth.config_volume("c2", seed=args.seed + rank, dtype=np.float32)
    u0_np = np.ascontiguousarray(u0_np, dtype=np.float32)
    phi0_np = np.ascontiguousarray(phi0_np, dtype=np.float32)
    dev = torch.device("cuda", local)
    u0_d = torch.from_numpy(u0_np).to(dev)
    phi0_d = torch.from_numpy(phi0_np).to(dev)
    phi_d = torch.empty_like(u0_d)
    u0_h = torch.from_numpy(u0_np).pin_memory()
    phi0_h = torch.from_numpy(phi0_np).pin_memory()
    phi_h = torch.empty(shape, dtype=torch.float32).pin_memory()

    ctx = pkg.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    kw = dict(PARAMS)
    kw["maxiter"] = wl["maxiter"]
    kw["sigma"] = wl["sigma"]
    if args.maxiter:
        kw["maxiter"] = args.maxiter
    params = pkg.default_params(**kw)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    stats = {}
    for _ in range(args.warmup):
        stats = ctx.rsfe_apply(u0_d, phi0_d, params, phi_out=phi_d)["stats"]

    # device-resident inputs: value
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    launches0 = ctx.launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    iters = 0
    sweeps = 0
    for _ in range(args.steps):
        stats = ctx.rsfe_apply(u0_d, phi0_d, params, phi_out=phi_d)["stats"]
        iters += stats["iterations"]
        sweeps += stats["total_sweeps"]
    ev1.record(stream)
    barrier()
    clocks = sampler.stop()
    launches = ctx.launches - launches0
    dt_ms = max_over_ranks(ev0.elapsed_time(ev1))
    total_vox_iters = sum_over_ranks(float(n) * iters)
    value = total_vox_iters / (dt_ms * 1e-3) / 1e9

    # end to end through the C ABI with pinned host buffers (H2D in, D2H out)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e_iters = 0
    for _ in range(args.steps):
        st = ctx.rsfe_apply(u0_h.numpy(), phi0_h.numpy(), params, phi_out=phi_h.numpy())["stats"]
        e_iters += st["iterations"]
    e1.record(stream)
    barrier()
    e_ms = max_over_ranks(e0.elapsed_time(e1))
    e_value = sum_over_ranks(float(n) * e_iters) / (e_ms * 1e-3) / 1e9

    # per-stage device time of one step (profiling pass, after the timed region); the
    # "poisson_solve" stage encloses the half-sweep and residual stages, so it is kept
    # out of the stage sums
    ctx.set_profiling(True)
    ctx.profile(reset=True)
    ctx.rsfe_apply(u0_d, phi0_d, params, phi_out=phi_d)
    prof = ctx.profile(reset=True)
    ctx.set_profiling(False)
    prof.pop("poisson_solve", None)

    # the half-sweep in its real launch sequence: per-launch events break the overlap of
    # consecutive (programmatically dependent) sweeps, so the dominant kernel is also
    # timed as the difference of a 202- and a 2-sweep solve on the same stream
    # (400 half-sweeps back to back; each solve has one residual check)
    sweep_us = half_sweep_us(ctx, shape, dev, stream) if rank == 0 else None

    result = None
    if rank == 0:
        peak, peak_kind = peaks()
        top = max(prof.items(), key=lambda kv: kv[1][0])
        name, (ms_total, count) = top
        avg_s = ms_total / count * 1e-3
        avg_s_events = avg_s
        if name == "rb_half" and sweep_us:
            avg_s = sweep_us * 1e-6
        per_vox = ALGO_BYTES_PER_VOXEL.get(name)
        achieved = per_vox * n / avg_s / 1e9 if per_vox else None
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic_per_voxel.json")
        if os.path.exists(tpath):
            tv = json.load(open(tpath)).get(name)
            if tv:
                traffic = float(tv["bytes_per_voxel"]) * n
        step_ms = prof_total = sum(v[0] for v in prof.values())
        roofline = {
            "bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "algo_bytes_per_launch": per_vox * n if per_vox else None,
            "avg_launch_us": avg_s * 1e6, "launches_per_step": count,
            "avg_launch_us_events": avg_s_events * 1e6,
            "launch_timing": ("back-to-back launches inside one solve (202- minus 2-sweep solve, "
                              "CUDA events on the library's stream)" if avg_s != avg_s_events
                              else "CUDA events around each launch in a profiled pass"),
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)",
            "share_of_step": ms_total / prof_total if prof_total else None,
        }
        # whole-iteration roofline: algorithmic bytes of every stage over the step time
        algo_step = sum(ALGO_BYTES_PER_VOXEL.get(k, 0.0) * n * c for k, (m, c) in prof.items())
        per_step_ms = dt_ms / args.steps
        roofline["step_algo_gb"] = algo_step / 1e9
        roofline["step_frac"] = (algo_step / (per_step_ms * 1e-3) / 1e9) / peak
        stages = {k: {"ms": round(v[0], 3), "launches": v[1],
                      "algo_gbs": (round(ALGO_BYTES_PER_VOXEL[k] * n * v[1] / (v[0] * 1e-3) / 1e9, 1)
                                   if k in ALGO_BYTES_PER_VOXEL and v[0] > 0 else None)}
                  for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
        # learned Poisson warm start (3-level 3x3x3 U-Net, 16/32/64 channels, 4 inputs):
        # an upper bound on its time-to-residual gain from measured numbers -- the plain
        # solve's device time per outer iteration against the network's FLOPs at the
        # measured dense bf16 peak, i.e. a perfect prediction (no sweeps after it) and a
        # network at 100 % of that peak; and the same bound with the network's time
        # measured on cuDNN's convolutions (random weights: the time does not depend on
        # them). The project builds no network of its own.
        solve_ms = 0.0
        for k, (m, c) in prof.items():
            if k == "rb_half":
                solve_ms += (sweep_us * 1e-3 * c) if sweep_us else m
            elif k == "rb_residual":
                solve_ms += m
        solve_ms_iter = solve_ms / max(kw["maxiter"], 1)
        unet_flop = unet_flop_estimate(shape)
        bf16, bf16_kind = bf16_peak_tflops()
        unet_ms = unet_flop / (bf16 * 1e12) * 1e3 if bf16 else None
        learned = {
            "plain_solve_ms_per_outer_iteration": solve_ms_iter,
            "unet_gflop_per_inference": unet_flop / 1e9,
            "bf16_peak_tflops": bf16,
            "bf16_peak_source": bf16_kind + " (MEASURED_PEAKS.json bf16_tflops, cuBLAS burst)",
            "unet_ms_at_peak": unet_ms,
            "speedup_upper_bound": (solve_ms_iter / unet_ms) if unet_ms else None,
            "target": 2.0,
            "note": "bound: a perfect prediction from a network at the measured bf16 peak",
        }
        # at N = 1 only, like the CPU baseline: the other ranks would wait at the final
        # barrier meanwhile
        if not args.no_unet and ws == 1:
            try:
                cu_ms = unet_forward_ms(shape, dev)
                learned["unet_ms_cudnn_bf16"] = cu_ms
                learned["speedup_upper_bound_cudnn"] = solve_ms_iter / cu_ms
                learned["unet_cudnn_tflops"] = unet_flop / (cu_ms * 1e-3) / 1e12
            except Exception as exc:  # the bound above stands without it
                learned["unet_cudnn_error"] = f"{type(exc).__name__}: {exc}"[:200]
            learned.update(learned_warm_start(pkg, ctx, shape, dev, stream, unet_flop, bf16))
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid volumes, one per rank)",
            "config": {"workload": (f"rsfe-sb {shape[0]}x{shape[1]}x{shape[2]} fp32, "
                                    f"{kw['maxiter']} outer iterations, RB-GS to rel. residual 1e-6"),
                       "shape": list(shape), "outer_iterations": kw["maxiter"],
                       "sigma": kw["sigma"], "volumes_per_rank": 1, "parallelism": f"replicas x{ws} (one volume per GPU)",
                       "l2": (f"every field {n * 4 / 2**20:.0f} MiB and each pass streams "
                              "several of them: inputs larger than the 126 MB L2, no flush"),
                       "gs_sweeps_per_step": sweeps / max(args.steps, 1)},
            "e2e": {"value": e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * n * 4,
                    "d2h_bytes_per_step": n * 4, "ms_per_step": e_ms / args.steps},
            "roofline": roofline, "stages_ms_per_step": stages, "gpu_launches": launches,
            "learned_warm_start_bound": learned,
            "clocks": clocks,
        }
        if args.workload != "c2":
            result["metric"] = METRIC.replace("@256^3", "@%dx%dx%d" % tuple(shape))
        if ws == 1 and not args.no_cpu and args.workload == "c2":
            result["cpu_baseline"] = cpu_baseline(args)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


# ------------------------------------------------------------ batched volumes
def run_batch(args):
    """48 volumes with sizes uniform in [96,256]x[96,256]x[64,192], each from the
    two-ellipsoid generator with its own seed, FP32, segmented by one batched call per
    step. Reports aggregate Gvoxel-iters/s and per-volume latency p50/p95."""
    import numpy as np
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    pkg = importlib.import_module("3dimagetoolkit_b200")
    shapes = pkg.synth.batch_shapes(48, seed=args.seed)
    shard = importlib.import_module("3dimagetoolkit_b200.shard")
    mine = shard.volume_shard(len(shapes), rank, ws)  # volumes shard across ranks
    dev = torch.device("cuda", local)
    vols, inits, outs = [], [], []
    for q in mine:
        u0 = pkg.synth.ellipsoids(shapes[q], 1000 + q, n=2, semi_axes=(8, 16), dtype=np.float32)
        vols.append(torch.from_numpy(np.ascontiguousarray(u0)).to(dev))
        inits.append(torch.from_numpy(pkg.synth.sphere_phi0(shapes[q], 20.0, dtype=np.float32)).to(dev))
        outs.append(torch.empty_like(vols[-1]))
    kw = dict(PARAMS)
    if args.maxiter:
        kw["maxiter"] = args.maxiter
    params = pkg.default_params(**kw)
    ctx = pkg.Context(local)
    mode = {"auto": pkg.BATCH_AUTO, "streams": pkg.BATCH_STREAMS, "worklist": pkg.BATCH_WORKLIST}[args.batch_mode]
    ctx.set_option(pkg.OPT_BATCH_MODE, mode)
    for _ in range(args.warmup):
        ctx.rsfe_apply_batched(vols, inits, params, streams=args.streams, outs=outs)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    launches0 = ctx.launches
    t0 = time.perf_counter()
    vox_iters = 0.0
    lats = []
    for _ in range(args.steps):
        _, stats, lat = ctx.rsfe_apply_batched(vols, inits, params, streams=args.streams, outs=outs)
        vox_iters += sum(float(v.numel()) * st["iterations"] for v, st in zip(vols, stats))
        lats.extend(lat)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    launches = ctx.launches - launches0
    vox_iters, dt = shard.job_throughput(vox_iters, dt)
    ctx.close()
    if rank == 0:
        line = {
            "metric": "RSFE-SB batched uneven volumes Gvoxel-iters/s (FP32, RB-GS to 1e-6)",
            "value": vox_iters / dt / 1e9, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (48 seeded two-ellipsoid volumes)",
            "config": {"workload": "48 volumes 96..256 x 96..256 x 64..192, 100 outer iterations",
                       "batch_mode": args.batch_mode, "streams": args.streams,
                       "volumes_per_rank": len(mine)},
            "latency_ms": {"p50": float(np.percentile(lats, 50)), "p95": float(np.percentile(lats, 95))},
            "gpu_launches": launches,
            "timing": "host wall clock around the batched calls (each call returns after all "
                      "its volumes are done)",
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


# ------------------------------------------------------------------ CPU arms
REF_FIXTURE = os.path.join(ROOT, "tests", "golden", "rsfe_c2_256_ref.npz")


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O

    return O


def _ref_fft(O, fft, threads) -> str:
    """The FFT behind the reference's FFTW calls: scipy's pocketfft (multi-threaded) or
    the in-tree FFT. Returns the one in use."""
    if fft == "pocketfft" and O.use_pocketfft(threads):
        return "scipy pocketfft behind the FFTW entry points (in place on the plan's output)"
    O.use_pocketfft(None)
    return "in-tree FP64 FFT behind the FFTW entry points"


def _ref_iterations(shape, maxiter, seed, threads, fft="pocketfft"):
    """Runs the reference's own code (FP64) on the 256^3 workload for maxiter outer
    iterations with `threads` OpenMP threads; returns, per outer iteration after the
    first, its wall seconds, the seconds inside its Poisson step and inside FFTs, and
    its sweeps, and the FFT used."""
    import numpy as np

    O = _oracle()
    O.set_threads(threads)
    used = _ref_fft(O, fft, threads)
    pkg = importlib.import_module("3dimagetoolkit_b200")
    u0, phi0 = pkg.synth.config_volume("c2", seed=seed, dtype=np.float64)
    kw = dict(PARAMS)
    kw["maxiter"] = maxiter
    O.rsfe_apply(u0, phi0, O.default_params(**kw), use_reference=True)
    ends = O.ref_last_timeline()[1:-1]  # end of each outer iteration's Poisson step
    marks = O.ref_last_sweep_marks()
    solve, fft = O.ref_last_step_profile()
    # iteration q runs from the end of step q-1 to the end of step q: the rest of
    # iteration q-1 (clamp, tolerance, Bregman, div) and the start and solve of q
    its = [{"seconds": float(ends[q] - ends[q - 1]), "solve": float(solve[q]),
            "fft": float(fft[q] - fft[q - 1]), "sweeps": float(marks[q] - marks[q - 1])}
           for q in range(1, len(ends))]
    O.use_pocketfft(None)
    return its, used


def _fftw_probe() -> str:
    import ctypes.util

    libs = [n for n in ("fftw3", "fftw3_omp", "fftw3_threads") if ctypes.util.find_library(n)]
    return ("found: " + ", ".join(libs)) if libs else "absent (no libfftw3 on this host)"


def _fft_seconds(threads):
    """One 274^3 complex FP64 transform (the size the reference's 256^3 convolutions
    pad to): the in-tree FFT behind the reference's FFTW calls, and scipy's pocketfft
    (ducc) with the same threads, for scale."""
    import numpy as np

    O = _oracle()
    O.set_threads(threads)
    O.use_pocketfft(None)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((274, 274, 274)) + 1j * rng.standard_normal((274, 274, 274))
    O.ref_fft3d(x)
    t0 = time.perf_counter()
    O.ref_fft3d(x)
    shim = time.perf_counter() - t0
    try:
        import scipy.fft

        scipy.fft.fftn(x, workers=threads)
        t0 = time.perf_counter()
        scipy.fft.fftn(x, workers=threads)
        ducc = time.perf_counter() - t0
    except ImportError:
        ducc = None
    return shim, ducc


def _ref_summary(its, threads, n, used):
    """The reference arm's figures from measured outer iterations."""
    import numpy as np

    tot = sum(r["seconds"] for r in its)
    solve = sum(r["solve"] for r in its)
    fft = sum(r["fft"] for r in its)
    sweeps = sum(r["sweeps"] for r in its)
    k = len(its)
    per_sweep = solve / max(sweeps, 1)
    out = {
        "value": n * k / tot / 1e9,
        "seconds_per_iteration": tot / k,
        "breakdown_s_per_iteration": {"fft": fft / k, "poisson_solve": solve / k,
                                      "other": (tot - fft - solve) / k},
        "sweeps_per_iteration": sweeps / k,
        "seconds_per_sweep": per_sweep,
        "threads": threads,
        "fftw": _fftw_probe(),
        "fft": used,
    }
    # The timed iterations are early ones; the full 100-iteration run (the GPU arm's
    # step) has its own sweep profile, recorded by the reference in the 256^3 fixture.
    if os.path.exists(REF_FIXTURE):
        d = np.load(REF_FIXTURE)
        s_full = float(d["total_sweeps"]) / float(d["iterations"])
        per_it = (tot - solve) / k + per_sweep * s_full
        out["same_profile"] = {
            "sweeps_per_iteration": s_full,
            "source": "the reference's own 100-iteration 256^3 run (tests/golden/rsfe_c2_256_ref.npz)",
            "seconds_per_iteration": per_it, "value": n / per_it / 1e9}
    return out


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(args):
    threads = args.ref_threads or os.cpu_count()
    t0 = time.time()
    its, used = _ref_iterations(SHAPE, 2, args.seed, threads, args.ref_fft)
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    summ = _ref_summary(its, threads, n, used)
    log(f"cpu baseline: {len(its)} timed iteration(s), {summ['seconds_per_iteration']:.2f} s each, "
        f"{time.time() - t0:.1f} s total")
    return {"value": summ["value"], "unit": UNIT, "cores": threads, "kind": "reference",
            "cpu_model": _cpu_model(), **{k: v for k, v in summ.items() if k != "value"},
            "sample": "reference C++ (oracle/_ref: the reference headers compiled with headless "
                      "VTK/GetPot shims; FFT as in `fft`), T=double, 256^3, wall time of outer "
                      "iteration 2 of 2 (setup and iteration 1 excluded)"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    threads = args.ref_threads or os.cpu_count()
    maxiter = 1 + args.warmup + args.steps
    its, used = _ref_iterations(SHAPE, maxiter, args.seed, threads, args.ref_fft)
    timed = its[args.warmup:args.warmup + args.steps] if len(its) > args.warmup else its
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    summ = _ref_summary(timed, threads, n, used)
    shim, ducc = _fft_seconds(threads)
    summ["fft_274cube_seconds"] = {"in_tree": shim, "scipy_pocketfft": ducc}
    value = summ.pop("value")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": len(timed), "warmup": args.warmup,
        "ms_per_step": summ["seconds_per_iteration"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded ellipsoid volume)",
        "config": {"workload": "rsfe-sb 256^3, one outer iteration per step, Poisson step solved "
                               "to rel. residual 1e-6 (red-black plug-in)", "shape": list(SHAPE)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "cpu_model": _cpu_model(), "host_cores": os.cpu_count(), **summ,
                         "sample": f"{len(timed)} outer iterations of the 256^3 workload after "
                                   f"{args.warmup} warm-up iterations and the set-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ref-threads", type=int, default=0,
                    help="OpenMP threads of the reference's CPU code (default: all host cores)")
    ap.add_argument("--ref-fft", default="pocketfft", choices=["pocketfft", "in-tree"],
                    help="FFT behind the reference's FFTW calls (no FFTW on these hosts): scipy's "
                         "pocketfft (default) or the in-tree FFT")
    ap.add_argument("--no-unet", action="store_true",
                    help="skip timing the library network behind the warm-start bound")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "batch"],
                    help="c2: one 256^3 volume per step (default); c3: 512x512x320 CT-like "
                         "volume, sigma 4, 200 iterations; batch: 48 uneven volumes")
    ap.add_argument("--streams", type=int, default=4, help="batch workload: concurrent streams")
    ap.add_argument("--batch-mode", default="auto", choices=["auto", "streams", "worklist"],
                    help="batch workload: stream queue (auto, the faster) or work list")
    ap.add_argument("--size", type=str, default="",
                    help="profiling only: cube side (256) or NX,NY,NZ of a smaller/larger case")
    ap.add_argument("--maxiter", type=int, default=0,
                    help="profiling only: outer iterations per step (default 100)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
