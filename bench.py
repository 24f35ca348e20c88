#!/usr/bin/env python
"""Benchmark of the B200 MPM workpiece step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config large|small|precision|batched|serving|precision_study]
                    [--instances M]

Workload (default `large`): the plain large single-instance step -- 256x128x128
cells, dx 0.02 mm, 8 particles/cell (~33.5M particles), Ti-6Al-4V, rounded
wedge tool, CFL 0.3.  A step is one MPM time step over every particle
(P2G with the Johnson-Cook return, grid update with the tool boundary, G2P).
Metric: particle-updates/s = live particles x K / device time of the K steps.
The working set (~7 GB of particle state per step) is far larger than the
126 MB L2, so no flush is needed between steps.

N > 1 (torchrun): every rank runs its own replica (the path does not shard a
single instance; replicas only, no data-path collective); the timing is the
max over ranks, value = total particle-updates / that time.

--config batched: the config-3 sweep (M = 512 uneven workpieces, 300 steps) in
one batch handle -- one persistent launch per step for all of them, launch shape
autotuned, step calls replayed from a CUDA graph -- reported beside the same
workpieces stepped one at a time through the plain handle (all of them, 20
steps each), as `plain_sequential` and `batched_over_plain`.

--config serving: the serving loop under Poisson arrivals (200 requests/s for
60 s, 16^3..96^3-cell requests at 8 ppc, 200-2000 steps, 150 GB budget):
throughput, p50/p99/p99.9 latency of the requests completed in the window,
offered/admitted/completed counts.

--config precision_study: config 4 (128x64x64 cells) for 1000 steps in FP64 and
(--repeats times) in FP32 from the same seeded state; relative errors of
momentum, kinetic + internal energy, peak von Mises stress, max temperature and
mean plastic strain, per FP32 run, median and worst.

--impl reference: the reference's own CUDA kernels (src/MPMSolver.cu, built from
its sources into oracle/_ref/) on the same workload -- rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import signal
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "edegpredict-engine-rotary_b200"))
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "particle-updates/s"
UNIT = "particle-updates/s"
# Algorithmic bytes per particle-update of the two-pass FP32 step (P2G pass
# 38 words read + 6 written, G2P pass 13 read + 25 written = 328 B), plus 56 B
# of plastic-state writes per yielding update and 48/ppc B of grid traffic.
B_ALG_BASE, B_ALG_YIELD, B_ALG_GRID = 328.0, 56.0, 48.0


def load_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(config: str):
    f = ROOT / "profiles" / "traffic.json"
    if f.exists():
        d = json.loads(f.read_text())
        v = d.get(config)
        if v:
            return float(v["bytes_per_launch"]), v.get("source", "")
    return None, ""


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"mpm_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.6)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.send_signal(signal.SIGINT)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        try:
            self.path.unlink()
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        load = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(n_gpus: int):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def physical_gpu_index(local: int) -> int:
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        ids = [x.strip() for x in cvd.split(",") if x.strip()]
        if local < len(ids) and ids[local].isdigit():
            return int(ids[local])
    return local


def make_case(name: str):
    from mpm_b200 import workpiece as W
    if name == "small":
        return W.config1(), "plain small: 64x32x32 cells, dx 0.05 mm, 8 ppc, AISI 4340, cylinder R 0.5 mm"
    if name == "precision":
        return W.config4(), "precision study geometry: 128x64x64 cells, dx 0.02 mm, 8 ppc, Ti-6Al-4V, wedge"
    if name == "cutting_precision":
        return W.config4(), ("cutting regime on the precision study geometry: 128x64x64 cells, dx 0.02 mm, 8 ppc, "
                             "Ti-6Al-4V, wedge at 2.5 m/s, timed after the engagement steps")
    if name == "cutting":
        return W.config2(), ("cutting regime on the plain large workload: 256x128x128 cells, dx 0.02 mm, 8 ppc "
                             "(~33.5M particles), Ti-6Al-4V, rounded wedge at 2.5 m/s, timed after the engagement "
                             "steps")
    return W.config2(), ("plain large single instance: 256x128x128 cells, dx 0.02 mm, 8 ppc (~33.5M particles), "
                         "Ti-6Al-4V, rounded wedge r_e 0.3 mm at 2.5 m/s, doc 0.05 mm, CFL 0.3")


# ----------------------------------------------------------------- CPU baseline

def cpu_baseline(case_name: str, budget_s: float = 15.0) -> dict:
    """The FP64 C restatement (oracle/) on the host cores, on a bounded sample
    of the workload: same material, tool and cell size, a 48x24x24-cell box."""
    from mpm_b200 import workpiece as W
    from oracle.oracle import Oracle
    o = Oracle()
    base, _ = make_case(case_name)
    cells = (48, 24, 24)
    if case_name == "small":
        case = W.config1(cells=cells)
    else:
        case = W.config2(cells=cells) if case_name == "large" else W.config4(cells=cells)
    st = W.full_state(W.generate_box(case), case)
    n_live = int((st["status"] != 1).sum())
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    st, _ = o.step(case, st, 1, nthreads=threads)
    t1 = time.perf_counter() - t0
    steps = max(1, min(200, int(budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    st, _ = o.step(case, st, steps, step0=1, t0=case["dt"], nthreads=threads)
    el = time.perf_counter() - t0
    return {"value": n_live * steps / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"FP64 C restatement (oracle/mpm_oracle.c, OpenMP) of the same step: {cells[0]}x{cells[1]}x"
                      f"{cells[2]} cells of the workload's material/tool/cell size ({n_live} particles), "
                      f"{steps} steps, {el:.1f} s"}


# ----------------------------------------------------------------- our arm

def run_ours(args):
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    from mpm_b200 import Solver, capi as A, workpiece as W
    case, desc = make_case(args.config)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    p = W.to_mpm_params(case)
    if args.contact_every > 0:
        # particle-side tool contact fused into the step (reference ContactConfig defaults)
        p.contact_every = int(args.contact_every)
    box = case["box"]
    T0 = box["T0"]
    if args.asb:
        # adiabatic shear band heating after the move (AdiabaticShearConfig defaults); the
        # workpiece starts 1 K above ambient so that every particle is past the model's
        # temperature guard and its strain-rate test decides
        p.asb_enabled = 1
        T0 = box["T0"] + 1.0
    if args.heat:
        # grid heat conduction (MPMWorkpieceSolver's scheme), reference default conductivity
        p.heat_conduction = 1
    cap = int(np.prod([box["c1"][i] - box["c0"][i] for i in range(3)]) * box["ppc"])
    s = Solver(p, cap, stream=stream.cuda_stream)
    if args.atomic or args.pass_size or args.ctas_per_sm or args.sort_every:
        s.set_launch_config(ctas_per_sm=args.ctas_per_sm or 4, sort_every=args.sort_every or 16,
                            deterministic=not args.atomic, pass_size=args.pass_size)
    launch_cfg = s.launch_config()
    n = s.init_box(box["c0"], box["c1"], box["ppc"], box["seed"] + rank, box["instance"], box["fixed_layers"],
                   T0, tool=case["tool"])
    m0 = s.metrics()
    n_live = n - m0["n_inactive"]
    dt = case["dt"]
    engage = args.engage_steps if args.config.startswith("cutting") else 0
    if engage:
        # the tool engages and chips form before the timed region (untimed)
        s.step(dt, engage)
        m0 = s.metrics()
        n_live = n - m0["n_inactive"]
    # warm-up (untimed)
    s.step(dt, args.warmup)
    torch.cuda.synchronize(dev)
    y0 = s.metrics()["n_yielded"]
    launches0 = s.launches()
    sampler = ClockSampler(physical_gpu_index(local))
    sampler.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    s.profile(True)
    s.profile_read()
    with torch.cuda.stream(stream):
        e0.record(stream)
        s.step(dt, args.steps)
        e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    k_ms, k_n = s.profile_read()
    s.profile(False)
    launches = s.launches() - launches0
    m1 = s.metrics()
    f_yield = (m1["n_yielded"] - y0) / max(1, n_live * args.steps)
    if dist:
        t = torch.tensor([ms, float(n_live)], device=dev, dtype=torch.float64)
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        tot = t.clone()
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        ms_max, live_tot = float(mx[0]), float(tot[1])
    else:
        ms_max, live_tot = ms, float(n_live)
    value = live_tot * args.steps / (ms_max / 1e3)

    peak, peak_kind = load_peaks()
    # end to end through the C ABI with host buffers (per replica)
    e2e = run_e2e(s, case, args, n, dev, stream)
    if dist:
        t = torch.tensor([e2e["seconds"]], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_val = live_tot * args.steps / float(t[0])
    else:
        e2e_val = float(n_live) * args.steps / e2e["seconds"]

    b_alg = B_ALG_BASE + B_ALG_YIELD * f_yield + B_ALG_GRID / box["ppc"]
    avg_launch_s = (k_ms / max(k_n, 1)) / 1e3
    achieved = b_alg * n_live / avg_launch_s / 1e9 if k_n else None
    traffic, traffic_src = load_traffic(args.config)
    s.close()
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_baseline("large" if args.config == "cutting" else
                               ("precision" if args.config == "cutting_precision" else args.config), args.cpu_seconds)
        variants = None
        plugin = None
        if world == 1 and args.config == "large" and not args.no_variants and not args.atomic:
            variants = like_for_like(case, args, dev, stream, peak)
            plugin = plugin_leg(case, args, dev)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "particles_per_gpu": int(n_live), "cells": list(case["cells"]),
                       "dx_m": case["params"]["dx"], "dt_s": dt, "ppc": box["ppc"],
                       "schedule": ("fused G2P->P2G, one kernel per step; node tiles added to the grid with "
                                    "FP32 atomics" if args.atomic else
                                    "fused G2P->P2G, one kernel per step; deterministic: stored node tiles "
                                    "summed per node in a fixed order (one node-sum launch per step)"),
                       "pass_size": launch_cfg["pass_size"], "sort_every": launch_cfg["sort_every"],
                       "ctas_per_sm": launch_cfg["ctas_per_sm"],
                       "parallelism": f"replicas{world}",
                       "l2": "working set >> L2 (no flush needed)", "yield_fraction": f_yield,
                       "escaped_updates": int(m1["n_escaped"]), "rebins": int(m1["n_sorts"]),
                       "contact_every": int(args.contact_every), "contacts": int(m1["n_contacts"]),
                       "adiabatic_shear": bool(args.asb), "asb_heated": int(m1["n_asb_heated"]),
                       "initial_rise_K": float(T0 - box["T0"]), "heat_conduction": bool(args.heat)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback",
                         "traffic": traffic, "traffic_source": traffic_src,
                         "kernel": "k_step<float,G2P,P2G> (fused)", "kernel_launches_timed": int(k_n),
                         "kernel_ms_avg": k_ms / max(k_n, 1), "bytes_alg_per_update": b_alg},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": e2e["h2d"] / args.steps,
                    "d2h_bytes_per_step": e2e["d2h"] / args.steps, "seconds": e2e["seconds"],
                    "path": e2e["path"]},
            "clocks": clocks,
        }
        if engage:
            out["config"]["engagement_steps"] = int(engage)
            out["config"]["chips"] = int(m1["n_chip"])
        if variants:
            out["like_for_like"] = variants
        if plugin:
            out["plugin"] = plugin
        if cpu:
            out["cpu_baseline"] = cpu
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def like_for_like(case, args, dev, stream, peak) -> dict:
    """The same workload with the reference's boundary and precision: the
    rasterised tool (surface samples of the wedge at half a cell, the
    reference's only grid boundary) in FP32, and in FP64 as the reference
    kernels compute.  Each line: particle-updates/s of one step call, the
    fused launch's average time and its fraction of the measured HBM peak
    (algorithmic bytes doubled in FP64)."""
    import torch
    from mpm_b200 import Solver, capi as A, workpiece as W
    box = case["box"]
    cap = int(np.prod([box["c1"][i] - box["c0"][i] for i in range(3)]) * box["ppc"])
    steps = max(10, min(args.steps, 60))
    out = {}
    for name, prec in (("raster_f32", A.PREC_F32), ("raster_f64", A.PREC_F64)):
        rc = dict(case)
        rc["tool"] = dict(case["tool"], mode=A.TOOL_RASTER)
        rc["tool"]["samples"] = W.tool_samples(rc)
        s = Solver(W.to_mpm_params(rc, precision=prec), cap, stream=stream.cuda_stream)
        try:
            s.set_tool(rc["tool"])
            n = s.init_box(box["c0"], box["c1"], box["ppc"], box["seed"], box["instance"], box["fixed_layers"],
                           box["T0"], tool=case["tool"])
            n_live = n - s.metrics()["n_inactive"]
            s.set_tool(rc["tool"])
            s.step(case["dt"], args.warmup)
            torch.cuda.synchronize(dev)
            y0 = s.metrics()["n_yielded"]
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            s.profile(True)
            s.profile_read()
            with torch.cuda.stream(stream):
                e0.record(stream)
                s.step(case["dt"], steps)
                e1.record(stream)
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1)
            k_ms, k_n = s.profile_read()
            s.profile(False)
            f_yield = (s.metrics()["n_yielded"] - y0) / max(1, n_live * steps)
        finally:
            s.close()
        b_alg = (B_ALG_BASE + B_ALG_YIELD * f_yield + B_ALG_GRID / box["ppc"]) * (2.0 if prec == A.PREC_F64 else 1.0)
        kms = k_ms / max(k_n, 1)
        achieved = b_alg * n_live / (kms / 1e3) / 1e9 if k_n else None
        out[name] = {"value": n_live * steps / (ms / 1e3), "unit": UNIT, "steps": steps,
                     "ms_per_step": ms / steps, "kernel_ms_avg": kms, "bytes_alg_per_update": b_alg,
                     "roofline_frac": (achieved / peak) if achieved else None, "samples": len(rc["tool"]["samples"]),
                     "tool": "raster (wedge surface samples at 0.5 cell)",
                     "dtype": "f64" if prec == A.PREC_F64 else "f32"}
    return out


def plugin_leg(case, args, dev) -> dict:
    """The same workload through the drop-in plugin (MPMSolverB200 via
    adapter/adapter_driver.cpp) in SimulationEngine's call pattern
    (src/SimulationEngine.cpp:495-536): per macro step setToolPosition,
    beginInterpolatedToolMotion on the FEM tool's device nodes (the wedge's
    surface samples at half a cell as FEMNodeGPU records, moving at the tool
    speed), eight interpolateToolForSubStep + step(dt), endInterpolatedToolMotion
    and syncMetrics (the metrics read back to the host).  Host-timed over the
    macro steps: every syncMetrics already waits for the device."""
    import torch
    from mpm_b200 import adapter as AD, capi as A, workpiece as W
    if not AD.available():
        return {"unavailable": "adapter driver not built (build.py --adapter with MPM_REFERENCE_SRC)"}
    box, tool = case["box"], case["tool"]
    cap = int(np.prod([box["c1"][i] - box["c0"][i] for i in range(3)]) * box["ppc"])
    sub = 8
    warm_m = max(1, -(-args.warmup // sub))
    timed_m = max(2, min(8, -(-args.steps // sub)))
    dt = case["dt"]
    smp = W.tool_samples(case)

    def pose(t):
        return [tool["position"][a] + tool["velocity"][a] * t for a in range(3)]

    nodes = [torch.from_numpy(AD.fem_node_records(smp + np.asarray(pose(m * sub * dt)), tool["velocity"]).copy())
             .to(dev) for m in range(warm_m + timed_m + 1)]
    ad = AD.Adapter(cap)
    try:
        ad.initialize(W.to_mpm_params(case))
        n = ad.seeded_box(box["c0"], box["c1"], box["ppc"], box["seed"], box["fixed_layers"], box["T0"], tool=tool)
        n_live = n - int(ad.sync_metrics()[1].n_inactive)

        def macro(m):
            ad.set_tool_position(pose(m * sub * dt))
            ad.begin_interp(nodes[m].data_ptr(), len(smp))
            for k in range(sub):
                ad.interp_substep(nodes[m + 1].data_ptr(), k / sub)
                ad.step(dt)
            ad.end_interp(nodes[m + 1].data_ptr())
            ad.sync_metrics()

        for m in range(warm_m):
            macro(m)
        ad.ok()
        torch.cuda.synchronize(dev)
        l0 = ad.launches()
        t0 = time.perf_counter()
        for m in range(warm_m, warm_m + timed_m):
            macro(m)
        sec = time.perf_counter() - t0
        ad.ok()
        launches = ad.launches() - l0
    finally:
        ad.close()
    steps = timed_m * sub
    return {"value": n_live * steps / sec, "unit": UNIT, "steps": steps, "ms_per_step": sec * 1e3 / steps,
            "launches_per_macro_step": launches / timed_m, "fem_nodes": len(smp),
            "d2h_bytes_per_macro_step": ctypes.sizeof(A.MpmMetrics) + 4 * 8,
            "dtype": "f32", "path": "MPMSolverB200 (IPhysicsSolver / IMetricsProvider drop-in): setToolPosition, "
                                    "beginInterpolatedToolMotion, 8 x (interpolateToolForSubStep + step), "
                                    "endInterpolatedToolMotion, syncMetrics"}


def run_e2e(s, case, args, n, dev, stream) -> dict:
    """Through the C ABI with host buffers: upload the particles from pinned
    host memory, step in macro steps of 8 sub-steps (set the tool pose, step,
    read the metrics, as SimulationEngine does), download the exported
    fields into pinned host memory."""
    import torch
    parts = s.download(fields=("x", "y", "z", "temperature", "status", "id"), elem=4)
    pin = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in parts.items()}
    outf = ("x", "y", "z", "vx", "vy", "vz", "stress", "temperature", "plastic_strain", "status")
    from mpm_b200 import capi as A
    out_bufs = {}
    for k in outf:
        per = A.PARTICLE_FIELDS.get(k, 1)
        dt_ = np.int32 if k == "status" else np.float32
        out_bufs[k] = torch.from_numpy(np.zeros((n, per) if per > 1 else (n,), dtype=dt_)).pin_memory().numpy()
    h2d = sum(v.nbytes for v in pin.values())
    d2h = sum(v.nbytes for v in out_bufs.values())
    tool = dict(case["tool"])
    dt = case["dt"]
    macro = 8
    # one untimed download sizes the handle's device staging buffer, as an
    # application's first download would: otherwise the timed region would
    # hold a one-time cudaMalloc of about 2 GB, whose cost varies by 10x
    s.download_into(out_bufs, elem=4)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    s.upload(pin, elem=4)
    done = 0
    while done < args.steps:
        k = min(macro, args.steps - done)
        s.set_tool(tool)
        s.step(dt, k)
        s.metrics()
        h2d += ctypes.sizeof(A.MpmToolDesc)
        d2h += ctypes.sizeof(A.MpmMetrics)
        done += k
    s.download_into(out_bufs, elem=4)
    torch.cuda.synchronize(dev)
    sec = time.perf_counter() - t0
    return {"seconds": sec, "h2d": h2d, "d2h": d2h,
            "path": "mpm_upload (pinned f32 SoA) -> per 8 sub-steps: mpm_set_tool + mpm_step + mpm_sync_metrics -> "
                    "mpm_download (pinned f32 SoA)"}


# ----------------------------------------------------------------- reference arm

# ----------------------------------------------------------------- batched arm

def _cap(case) -> int:
    b = case["box"]
    return int(np.prod([b["c1"][i] - b["c0"][i] for i in range(3)]) * b["ppc"])


def _init(obj, case, i=None, rank=0):
    b = case["box"]
    args = (b["c0"], b["c1"], b["ppc"], b["seed"] + rank, b["instance"], b["fixed_layers"], b["T0"])
    if i is None:
        return obj.init_box(*args, tool=case["tool"])
    return obj.init_box_i(i, *args, tool=case["tool"])


def plain_sequential(cases, steps: int, stream) -> dict:
    """The same workpieces one at a time through the plain single-instance
    handle (mpm_create / mpm_step), each timed with CUDA events on its stream."""
    import torch
    from mpm_b200 import Solver, workpiece as W
    tot_pu, tot_ms = 0.0, 0.0
    for c in cases:
        s = Solver(W.to_mpm_params(c), _cap(c), stream=stream.cuda_stream)
        n = _init(s, c)
        s.step(c["dt"], 3)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            s.step(c["dt"], steps)
            e1.record(stream)
        torch.cuda.synchronize()
        tot_ms += e0.elapsed_time(e1)
        tot_pu += n * steps
        s.close()
    return {"value": tot_pu / (tot_ms / 1e3), "unit": UNIT, "instances": len(cases), "steps": steps}


def run_batched(args):
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    from mpm_b200 import Batch, workpiece as W
    cases = W.config3(args.instances, seed=7 + rank)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    bt = Batch([W.to_mpm_params(c) for c in cases], [_cap(c) for c in cases], stream=stream.cuda_stream)
    n_live = 0
    for i, c in enumerate(cases):
        n_live += _init(bt, c, i, rank)
    dts = [c["dt"] for c in cases]
    # autotune (real steps, untimed) then warm-up
    if args.atomic:
        bt.set_launch_config(deterministic=False)
    tune = bt.autotune(dts) if not args.no_tune else bt.launch_config()
    bt.set_launch_config(tune["ctas_per_sm"], tune["sort_every"], use_graph=True, pass_size=tune["pass_size"],
                         deterministic=not args.atomic)
    tune = bt.launch_config()
    bt.step_all(dts, args.warmup)
    torch.cuda.synchronize(dev)
    launches0 = bt.launches()
    sampler = ClockSampler(physical_gpu_index(local))
    sampler.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        bt.step_all(dts, args.steps)
        e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = bt.launches() - launches0
    # kernel time of the fused launches (separate pass of the same length, not graph-replayed)
    bt.set_launch_config(tune["ctas_per_sm"], tune["sort_every"], use_graph=False, pass_size=tune["pass_size"],
                         deterministic=not args.atomic)
    bt.profile(True)
    bt.profile_read()
    bt.step_all(dts, min(args.steps, 50))
    k_ms, k_n = bt.profile_read()
    bt.profile(False)
    yielded = bt.metrics_i(0)["n_yielded"]   # the counter covers every instance of the handle
    bt.close()
    if dist:
        t = torch.tensor([ms, float(n_live)], device=dev, dtype=torch.float64)
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        tot = t.clone()
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        ms_max, live_tot = float(mx[0]), float(tot[1])
    else:
        ms_max, live_tot = ms, float(n_live)
    value = live_tot * args.steps / (ms_max / 1e3)
    out = None
    if rank == 0:
        sample = cases   # every workpiece of the batch, each alone
        plain = plain_sequential(sample, 20, stream)
        peak, peak_kind = load_peaks()
        ppc_mean = float(np.mean([c["box"]["ppc"] for c in cases]))
        steps_total = args.steps + args.warmup + (0 if args.no_tune else 168) + min(args.steps, 50)
        f_yield = yielded / max(1.0, n_live * steps_total)
        b_alg = B_ALG_BASE + B_ALG_YIELD * f_yield + B_ALG_GRID / ppc_mean
        avg = (k_ms / max(k_n, 1)) / 1e3
        achieved = b_alg * n_live / avg / 1e9 if k_n else None
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": f"batched: {len(cases)} workpieces of the config-3 sweep (cells log-uniform "
                                      "16^3..64^3, aspect 1-4, 4-8 ppc, per-instance Johnson-Cook, speed and depth "
                                      "of cut, rounded-wedge tool), one persistent launch per step, CUDA graph",
                          "instances": len(cases), "particles_per_gpu": int(n_live), "launch_config": tune,
                          "parallelism": f"replicas{world}", "l2": "working set >> L2 (no flush needed)",
                          "yield_fraction": f_yield},
               "gpu_launches": int(launches),
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": (achieved / peak) if achieved else None,
                            "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                            else "fallback", "traffic": None,
                            "kernel": "k_step<float,G2P,P2G> (fused)", "kernel_launches_timed": int(k_n),
                            "kernel_ms_avg": k_ms / max(k_n, 1), "bytes_alg_per_update": b_alg},
               "plain_sequential": dict(plain, sample=f"all {len(sample)} workpieces of the batch, one at a time "
                                                      "through mpm_create/mpm_step, 20 timed steps each"),
               "batched_over_plain": value / plain["value"],
               "clocks": clocks}
    if dist:
        dist.barrier()
    return out


# ----------------------------------------------------------------- precision study

def run_precision_study(args):
    """Config 4: the same workpiece stepped in FP32 (the product) and in FP64
    (the oracle run of the same kernels) from the same seeded state; relative
    errors of the conservation and peak quantities after K steps, for several
    seeds of the placement.  With the default deterministic node sums every
    FP32 run gives the same bits (--atomic: they vary in the last bits).  The
    fracture zone under the tool edge makes threshold decisions (damage, chip
    separation, the chip-fracture velocity kick) that can fall differently in
    FP32 and FP64 for a particle close to a threshold; each seed reports how
    many particles end with another status."""
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    from mpm_b200 import Solver, capi as A, workpiece as W
    seeds = [int(v) for v in args.seeds.split(",")]
    fields = ("x", "y", "z", "vx", "vy", "vz", "plastic_strain", "temperature", "stress", "status")

    def rel(x, y):
        return abs(x - y) / max(abs(y), 1e-300)

    per_seed, t64s, t32 = [], [], []
    n = 0
    for seed in seeds:
        case = W.config4()
        case["box"]["seed"] = seed
        b = case["box"]
        cap = int(np.prod([b["c1"][i] - b["c0"][i] for i in range(3)]) * b["ppc"])

        def run(prec):
            s = Solver(W.to_mpm_params(case, precision=prec), cap)
            s.set_launch_config(deterministic=not args.atomic)
            n = _init(s, case, rank=rank)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.step(case["dt"], args.steps)
            m = s.metrics()
            sec = time.perf_counter() - t0
            state = s.download(fields)      # generation order: the same particles in both precisions
            s.close()
            return n, m, sec, state

        n, r, t64, st64 = run(A.PREC_F64)
        t64s.append(t64)
        e64 = r["kinetic"] + r["internal_elastic"]
        a_tamb = case["params"]["Tamb"]
        vt = float(np.linalg.norm(case["tool"]["velocity"]))
        live = st64["status"] != A.INACTIVE
        v64 = np.sqrt(st64["vx"] ** 2 + st64["vy"] ** 2 + st64["vz"] ** 2)
        scales = {"position": case["params"]["dx"], "velocity": max(float(v64[live].max()), vt),
                  "plastic_strain": max(float(st64["plastic_strain"][live].max()), 1e-30),
                  "temperature_rise": max(float((st64["temperature"][live] - a_tamb).max()), 1e-30),
                  "stress": max(float(np.abs(st64["stress"][live]).max()), 1e-30)}

        def particle_errors(st):
            """Per-particle |FP32 - FP64| over the field scales: max and 99th percentile."""
            d = {"position": np.sqrt((st["x"] - st64["x"]) ** 2 + (st["y"] - st64["y"]) ** 2 +
                                     (st["z"] - st64["z"]) ** 2),
                 "velocity": np.sqrt((st["vx"] - st64["vx"]) ** 2 + (st["vy"] - st64["vy"]) ** 2 +
                                     (st["vz"] - st64["vz"]) ** 2),
                 "plastic_strain": np.abs(st["plastic_strain"] - st64["plastic_strain"]),
                 "temperature_rise": np.abs(st["temperature"] - st64["temperature"]),
                 "stress": np.abs(st["stress"] - st64["stress"]).max(axis=1)}
            return {k: {"max": float(v[live].max() / scales[k]), "p99": float(np.quantile(v[live], 0.99) / scales[k])}
                    for k, v in d.items()}

        def errors(a, st32):
            p32, p64 = np.array(a["momentum"]), np.array(r["momentum"])
            return {"momentum": float(np.linalg.norm(p32 - p64) / max(np.linalg.norm(p64), 1e-300)),
                    "kinetic_plus_internal": rel(a["kinetic"] + a["internal_elastic"], e64),
                    "peak_von_mises": rel(a["max_von_mises"], r["max_von_mises"]),
                    "max_temperature_rise": rel(a["max_temperature"] - a_tamb, r["max_temperature"] - a_tamb),
                    "mean_plastic_strain": rel(a["mean_plastic_strain"], r["mean_plastic_strain"]),
                    "n_chip": [a["n_chip"], r["n_chip"]], "n_yielded": [a["n_yielded"], r["n_yielded"]],
                    "status_differs": int((st32["status"] != st64["status"]).sum()),
                    "particles": particle_errors(st32)}
        runs = []
        for _ in range(max(1, args.repeats)):
            _, a, sec, st32 = run(A.PREC_F32)
            runs.append(errors(a, st32))
            t32.append(sec)
            del st32
        per_seed.append({"seed": seed, "runs": runs})
    if rank != 0:
        return None
    keys = ("momentum", "kinetic_plus_internal", "peak_von_mises", "max_temperature_rise", "mean_plastic_strain")
    first = [x["runs"][0] for x in per_seed]          # one FP32 result per seed (deterministic)
    med = {k: float(np.median([x[k] for x in first])) for k in keys}
    worst = {k: max(x[k] for x in first) for k in keys}
    within = [x["seed"] for x in per_seed if x["runs"][0]["momentum"] <= 1e-4
              and x["runs"][0]["kinetic_plus_internal"] <= 1e-4]
    flips = [x["seed"] for x in per_seed if x["runs"][0]["status_differs"] > 0]
    agree = [x["runs"][0] for x in per_seed if x["runs"][0]["status_differs"] == 0]
    repeat_same = all(all(r["momentum"] == x["runs"][0]["momentum"] for r in x["runs"]) for x in per_seed)
    return {"metric": "relative error FP32 vs FP64 after K steps (median over the seeds)",
            "value": max(med["momentum"], med["kinetic_plus_internal"]), "unit": "relative", "n_gpus": 1,
            "steps": args.steps, "warmup": 0, "ms_per_step": None, "higher_is_better": False, "scaling": None,
            "vs_baseline": None, "dtype": "f32 vs f64", "data": "synthetic",
            "config": {"workload": "precision study: 128x64x64 cells, dx 0.02 mm, 8 ppc, Ti-6Al-4V, rounded wedge "
                                   "r_e 0.3 mm at 2.5 m/s, doc 0.05 mm; the Johnson-Cook Newton solve and the "
                                   "conservation reductions are FP64 in both runs",
                       "particles": int(n), "seeds": seeds, "fp32_runs_per_seed": max(1, args.repeats),
                       "deterministic": not args.atomic,
                       "target": "momentum and kinetic+internal energy within 1e-4"},
            "errors_median": med, "errors_worst": worst, "seeds_within_1e-4": within,
            "seeds_with_status_flips": flips,
            "errors_worst_without_flips": {k: (max(x[k] for x in agree) if agree else None) for k in keys},
            "fp32_repeats_identical": repeat_same, "per_seed": per_seed,
            "wall_s": {"f64_each": t64s, "f32_each": t32}}


# ----------------------------------------------------------------- serving arm

def run_serving(args):
    """Continuous batching under Poisson arrivals: a submitter thread submits
    each request at its arrival time (the server stamps it then) while this
    thread runs the server's ticks; after the window, throughput = particle
    updates done in the window / its length, latency = done - submit of the
    requests that completed in it."""
    import threading
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    from mpm_b200 import Server, capi as A, workpiece as W
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    rng = np.random.default_rng(17 + rank)
    n_arr = int(args.rate * args.duration * 1.5) + 16
    gaps = rng.exponential(1.0 / args.rate, n_arr)
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < args.duration]
    reqs = []
    for i in range(len(arrivals)):
        c = W.config3_case(rng, i, cells_lo=16, cells_hi=96, ppc=8)
        reqs.append((c, int(rng.integers(200, 2001))))
    srv = Server(precision=A.PREC_F32, hbm_budget_bytes=int(args.budget_gb * 1e9), max_chunk=args.chunk,
                 use_graph=True, stream=stream.cuda_stream, max_resident_particles=int(args.resident_particles))
    ids = []
    stop = threading.Event()

    def submitter(t0):
        for k, (c, n) in enumerate(reqs):
            delay = t0 + arrivals[k] - time.perf_counter()
            if delay > 0 and stop.wait(delay):
                return
            ids.append(srv.submit(c, n))

    sampler = ClockSampler(physical_gpu_index(local))
    sampler.start()
    t0 = time.perf_counter()
    th = threading.Thread(target=submitter, args=(t0,), daemon=True)
    th.start()
    ticks = 0
    while time.perf_counter() - t0 < args.duration:
        if srv.tick() == 0:
            time.sleep(0.001)
        ticks += 1
    elapsed = time.perf_counter() - t0
    stop.set()
    th.join()
    st = srv.stats()
    clocks = sampler.stop()
    lat, done_particles = [], 0
    for i in list(ids):
        r = srv.poll(i)
        if r["state"] == A.REQ_DONE and r["t_done"] <= elapsed:
            lat.append(r["t_done"] - r["t_submit"])
            done_particles += r["n_particles"] * r["steps_done"]
    srv.close()
    value = st["particle_updates"] / elapsed
    out = None
    if rank == 0:
        sample = [c for c, _ in reqs[:16]]
        plain = plain_sequential(sample, 20, stream)
        q = (lambda p: float(np.percentile(lat, p))) if lat else (lambda p: None)
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": None,
               "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic",
               "config": {"workload": f"serving: Poisson arrivals at {args.rate:g} requests/s for {args.duration:g} s, "
                                      "requests of 16^3..96^3 cells (log-uniform, aspect 1-4) at 8 ppc, parameters as "
                                      "the config-3 sweep, 200-2000 steps each; continuous batching, state resident "
                                      f"on the device, admission by a {args.budget_gb:g} GB budget, chunks of "
                                      f"{args.chunk} steps per tick",
                          "parallelism": f"replicas{world}", "budget_gb": args.budget_gb, "max_chunk": args.chunk,
                          "max_resident_particles": int(args.resident_particles)},
               "requests": {"offered": st["offered"], "admitted": st["admitted"], "completed_in_window": len(lat),
                            "queued_at_end": st["queued"], "resident_at_end": st["resident"],
                            "resident_particles_at_end": st["resident_particles"], "ticks": st["ticks"]},
               "latency_s": {"p50": q(50), "p99": q(99), "p999": q(99.9), "of": "requests completed in the window"},
               "completed_particle_updates_per_s": done_particles / elapsed,
               "plain_sequential": dict(plain, sample="the first 16 requests, one at a time through mpm_create/"
                                                      "mpm_step, 20 timed steps each"),
               "served_over_plain": value / plain["value"],
               "clocks": clocks}
    if dist:
        dist.barrier()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    try:
        from oracle.oracle import RefKern
        from mpm_b200 import workpiece as W
        rk = RefKern()
    except Exception as exc:  # the harness was not built here
        return {"impl": "reference", "unavailable": f"reference kernels not built: {exc}"}
    import torch
    torch.cuda.set_device(0)
    if args.config == "batched":
        return run_reference_batched(args, rk)
    if args.config == "serving":
        return run_reference_serving(args, rk)
    case, desc = make_case(args.config)
    x, y, z, status = W.generate_box_chunked(case)
    samples = W.tool_samples(case)
    ms, live = rk.bench_positions(case, x, y, z, status, args.warmup, args.steps, samples=samples)
    n_live = int((status != 1).sum())
    value = n_live * args.steps / (ms / 1e3)
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "particles_per_gpu": n_live, "tool_boundary": "rasterised tool samples "
                       "(rasterizeToolKernel), the reference's only grid tool boundary"},
            "cpu_baseline": {"value": value, "unit": UNIT, "kind": "reference", "cores": 0,
                             "sample": "the reference has no CPU implementation of this path; its own CUDA kernels "
                                       "(src/MPMSolver.cu, FP64 AoS, CUDA graph per step as MPMSolver::step) on the "
                                       "B200, full workload"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _ref_line(value, desc, extra, sample):
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": None,
            "warmup": None, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": dict({"workload": desc}, **extra),
            "cpu_baseline": {"value": value, "unit": UNIT, "kind": "reference", "cores": 0, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _ref_instance(rk, case, warmup, steps):
    """One workpiece alone through the reference kernels (FP64 AoS, a CUDA
    graph per step as MPMSolver::step, the rasterised tool): device ms of
    `steps` steps and live particles."""
    from mpm_b200 import workpiece as W
    x, y, z, status = W.generate_box_chunked(case)
    ms, live = rk.bench_positions(case, x, y, z, status, warmup, steps, samples=W.tool_samples(case))
    return ms, int((status != 1).sum())


def run_reference_batched(args, rk):
    """The config-3 sweep as the reference runs it: one MPMSolver per
    workpiece, one after another (it has no batched form).  A bounded sample:
    workpieces in sweep order, 20 timed steps each, until about 60 s of work;
    value = their particle updates / their summed device time."""
    from mpm_b200 import workpiece as W
    cases = W.config3(args.instances, seed=7)
    steps = min(args.steps, 20)
    t_start = time.perf_counter()
    pu, ms_tot, k = 0.0, 0.0, 0
    for c in cases:
        ms, live = _ref_instance(rk, c, 2, steps)
        pu += live * steps
        ms_tot += ms
        k += 1
        if time.perf_counter() - t_start > 60.0:
            break
    value = pu / (ms_tot / 1e3)
    return _ref_line(value, "batched: the config-3 sweep (512 workpieces, cells log-uniform 16^3..64^3, aspect 1-4, "
                            "4-8 ppc, per-instance Johnson-Cook, speed and depth of cut, rounded-wedge tool), each "
                            "workpiece alone through the reference kernels, one after another",
                     {"instances": len(cases), "instances_timed": k, "steps_per_instance": steps},
                     f"the reference has no CPU implementation of this path; its own CUDA kernels (src/MPMSolver.cu, "
                     f"FP64 AoS, CUDA graph per step) on the B200: the first {k} workpieces of the sweep, "
                     f"{steps} timed steps each")


def run_reference_serving(args, rk):
    """The serving workload as the reference would serve it: requests in
    arrival order (FIFO), one MPMSolver at a time.  Each request's service
    time is the reference kernels' device time for its steps, measured on
    min(steps, 50) steps and scaled to its step count; the queue is then
    played over the window with the same Poisson arrivals as our arm:
    throughput = particle updates done in the window / the window,
    latency = completion - arrival of the requests completed in it."""
    from mpm_b200 import workpiece as W
    rng = np.random.default_rng(17)
    n_arr = int(args.rate * args.duration * 1.5) + 16
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, n_arr))
    arrivals = arrivals[arrivals < args.duration]
    reqs = []
    for i in range(len(arrivals)):
        c = W.config3_case(rng, i, cells_lo=16, cells_hi=96, ppc=8)
        reqs.append((c, int(rng.integers(200, 2001))))
    clock, done_pu, lat, k = 0.0, 0.0, [], 0
    t_start = time.perf_counter()
    for (c, n), t_arr in zip(reqs, arrivals):
        if clock >= args.duration or time.perf_counter() - t_start > 120.0:
            break
        meas = min(n, 50)
        ms, live = _ref_instance(rk, c, 2, meas)
        service = ms / 1e3 * n / meas
        start = max(clock, t_arr)
        end = start + service
        frac = min(1.0, max(0.0, (args.duration - start) / service))
        done_pu += live * n * frac
        if end <= args.duration:
            lat.append(end - t_arr)
        clock = end
        k += 1
    q = (lambda p: float(np.percentile(lat, p))) if lat else (lambda p: None)
    out = _ref_line(done_pu / args.duration,
                    f"serving: Poisson arrivals at {args.rate:g} requests/s for {args.duration:g} s, requests of "
                    "16^3..96^3 cells at 8 ppc, 200-2000 steps, served first come first served by the reference "
                    "kernels one request at a time",
                    {"requests_offered": len(reqs), "requests_started": k, "completed_in_window": len(lat)},
                    "the reference has no CPU implementation of this path; its own CUDA kernels (src/MPMSolver.cu, "
                    "FP64 AoS, CUDA graph per step) on the B200: each request's service time measured on "
                    "min(steps, 50) steps and scaled to its steps, played in arrival order over the window")
    out["latency_s"] = {"p50": q(50), "p99": q(99), "p999": q(99.9), "of": "requests completed in the window"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="large", choices=["large", "small", "precision", "batched", "serving",
                                                           "precision_study", "cutting", "cutting_precision"])
    ap.add_argument("--engage-steps", type=int, default=1000,
                    help="cutting configs: untimed steps before the timed region (the tool engages, chips form)")
    ap.add_argument("--no-variants", action="store_true",
                    help="large config: skip the like-for-like lines (raster tool FP32, raster tool FP64)")
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--contact-every", type=int, default=0,
                    help="plain configs: fuse the particle-side tool contact every n steps (0: off)")
    ap.add_argument("--asb", action="store_true",
                    help="plain configs: run the adiabatic shear band heating after every move")
    ap.add_argument("--heat", action="store_true",
                    help="plain configs: grid heat conduction (scatter, diffusion step, gather) every step")
    ap.add_argument("--repeats", type=int, default=2,
                    help="precision_study: FP32 runs per seed (identical unless --atomic)")
    ap.add_argument("--seeds", default="1234,1,2,3,4,6,8,9",
                    help="precision_study: placement seeds, comma-separated")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: requests per second")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: window in seconds")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: HBM budget")
    ap.add_argument("--chunk", type=int, default=50, help="serving: steps per tick at most")
    ap.add_argument("--resident-particles", type=float, default=0,
                    help="serving: admission cap on resident particles (0: the HBM budget alone)")
    ap.add_argument("--ctas-per-sm", type=int, default=0,
                    help="plain configs: persistent CTAs per SM of the step kernel (0: the default, 4)")
    ap.add_argument("--sort-every", type=int, default=0,
                    help="plain configs: steps between re-bins (0: the default, 16)")
    ap.add_argument("--pass-size", type=int, default=0, choices=[0, 128, 256, 512],
                    help="plain configs: FP32 particles per pass of the step kernel (0: the default)")
    ap.add_argument("--atomic", action="store_true",
                    help="plain configs and precision_study: add node tiles with FP32 atomics instead of the "
                         "default deterministic node sums")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps is None:
        args.steps = {"batched": 300, "precision_study": 1000}.get(args.config, 500)
    if args.impl == "reference":
        out = run_reference(args)
    elif args.config == "batched":
        out = run_batched(args)
    elif args.config == "serving":
        out = run_serving(args)
    elif args.config == "precision_study":
        out = run_precision_study(args)
    else:
        out = run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
