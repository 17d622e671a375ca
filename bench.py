#!/usr/bin/env python
"""Benchmark of the D3Q27 cumulant level step on B200.

Workload (one GPU): the 256 x 128 x 128 sphere channel (D = 24 cells at x = 64, inlet u = 0.05,
Re = 1000, zero-gradient outlet, lateral mirrors, half-way bounce-back with the FP64
momentum-exchange drag collected every step), FP32 arithmetic, populations stored as FP16
deviations from the lattice weights. A step is one fused pull-stream-collide launch over all
8,192 blocks plus the deterministic FP64 drag reduction.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--storage f16|f32|bf16|f64]

MLUPS counts every cell of the level, like the reference (src/main.jl:1265,1698-1712). With N > 1
each rank runs an independent replica (the step is not domain-decomposed here), so per-GPU work
is fixed and ``value`` is the aggregate over ranks (weak scaling).

``--impl reference`` times the reference's algorithm on the host cores: the CPU restatement of
the reference's Julia kernel (the reference itself is Julia and cannot run on this image), FP32,
OpenMP over every host thread, on a bounded sample of the same workload.
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
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS & % of HBM roofline; batched/served vs plain cases/s; p50/p99 latency"
STORAGE_BYTES = {"f16": 2, "bf16": 2, "f32": 4, "f64": 8}


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def traffic_record(storage):
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "cumulant_d3q27_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    rec = d.get(storage)
    return None if rec is None else rec.get("dram_bytes_per_launch")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms while the sampler is open; the
    timed region starts only after the first sample has been written."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            self.file.flush()
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        loaded = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------------------------
# CPU arm (the reference's algorithm on the host cores)
# ---------------------------------------------------------------------------------------------
def cpu_sample_case():
    """Bounded sample of the workload: a 256 x 128 x 16 slab of the channel (same inlet, outlet,
    mirror faces and sphere centre line, sphere cut by the slab), 524,288 cells, built by the
    oracle's own block builder and sphere mask (the product library is not loaded)."""
    import oracle
    return oracle.sphere_channel(256, 128, 16, diameter=24.0, centre_x=64.0)


def run_cpu_arm(steps, warmup, target_s=None):
    """Time the FP32 oracle on every host thread; returns (MLUPS, cores, steps_done, seconds)."""
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    case = cpu_sample_case()
    O = case.level(np.float32)
    p = case.params
    for _ in range(warmup):
        O.step(p)
    t0 = time.perf_counter()
    done = 0
    while True:
        O.step(p)
        done += 1
        el = time.perf_counter() - t0
        if target_s is None and done >= steps:
            break
        if target_s is not None and (el >= target_s or done >= steps):
            break
    el = time.perf_counter() - t0
    cells = case.n_blocks * 512
    return cells * done / el / 1e6, cores, done, el, cells


def reference_arm(args, rank, world):
    if rank != 0:
        return
    mlups, cores, done, el, cells = run_cpu_arm(args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * el / done, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.storage),
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
                         "sample": f"{cells} cells/step: 256x128x16 slab of the channel, FP32 C++ restatement of "
                                   "kernel_cumulant.jl (Julia reference not runnable here)"},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(storage, nz=128):
    return {"workload": f"sphere_channel_256x128x{nz}_D24_Re1000", "cells": 256 * 128 * nz, "blocks": 32 * 16 * (nz // 8),
            "operator": "cumulant_d3q27", "storage": f"{storage}_dev" if storage in ("f16", "bf16") else storage,
            "c_wale": 0.2, "solid_bc": "halfway", "forces": "FP64 momentum exchange every step",
            "l2": "inputs larger than L2 (populations 2 x %d MB)" % (256 * 128 * nz * 27 * STORAGE_BYTES[storage] // 2**20),
            "parallelism": "replicas"}


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f16", choices=["f16", "bf16", "f32", "f64"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU-baseline leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--nz", type=int, default=128, help="channel depth (smaller values for profiling captures)")
    ap.add_argument("--layout", default="block", choices=["block", "dense"], help="population layout of the level")
    ap.add_argument("--q19-steps", type=int, default=100,
                    help="steps of the D3Q19 octree periodic-box measurement (256^3, FP32 and FP64); 0 skips it")
    ap.add_argument("--kbc-steps", type=int, default=20,
                    help="steps of the D3Q39 entropic KBC measurement (128^3 periodic Taylor-Green, FP32); 0 skips it")
    ap.add_argument("--batch-steps", type=int, default=2000,
                    help="steps of the batched-vs-plain-loop comparison (64-case config 4); 0 skips it")
    ap.add_argument("--steady-seconds", type=float, default=1.0,
                    help="length of the steady-state pass timed after the K steps (clock record and MLUPS)")
    ap.add_argument("--tgv-steps", type=int, default=1000,
                    help="steps of the 64^3 FP64 Taylor-Green accuracy run (config 1); 0 skips it")
    ap.add_argument("--drag-steps", type=int, default=20000,
                    help="steps of the config-2 drag accuracy run per storage (FP64, FP32, FP16, BF16); 0 skips it")
    ap.add_argument("--drag-avg", type=int, default=5000, help="steps the drag coefficient is averaged over")
    ap.add_argument("--serve-requests", type=int, default=24,
                    help="requests of the served-vs-sequential comparison (config 5 mix); 0 skips it")
    ap.add_argument("--serve-steps", type=int, default=2000, help="steps per served request")
    ap.add_argument("--serve-kbc-share", type=float, default=0.25, help="fraction of D3Q39 KBC requests served")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the launch autotuner (oal_level_autotune) before the warm-up")
    ap.add_argument("--prefetch", type=int, default=-1,
                    help="set the x-pair kernel's L2 prefetch distance (CTAs) instead of autotuning it")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    # CPU leg first (before any CUDA call), rank 0 at N = 1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        mlups, cores, done, el, cells = run_cpu_arm(10**6, 1, target_s=args.cpu_seconds)
        cpu = {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
               "sample": f"{done} steps of {cells} cells (256x128x16 slab of the channel), FP32 C++ restatement "
                         f"of kernel_cumulant.jl, OpenMP {cores} threads, {el:.1f} s"}

    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()

    from openaerolab_alpha_01_b200 import _capi as capi
    from openaerolab_alpha_01_b200.cases import sphere_channel_case
    from openaerolab_alpha_01_b200.solver import Geometry, Level

    case = sphere_channel_case(256, 128, args.nz, diameter=24.0, centre_x=64.0)
    geom = Geometry(case.dom, device=dev)
    level = Level(geom, storage=args.storage, layout=args.layout)
    level.init_equilibrium(case.rho, case.vel)
    p = case.params
    cells = case.dom.n_blocks * 512
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()

    # the project's autotuner picks the x-pair kernel's L2 prefetch distance on this workload; it
    # restores the level's state, so the warm-up and the timed steps start from the initial state
    if args.prefetch >= 0:
        level.prefetch_ctas = args.prefetch
        tuning = {"prefetch_ctas": args.prefetch, "candidates": None}
    else:
        tuning = None if args.no_autotune else level.autotune(p, 20)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            p.time_step_seed = i
            level.perform_timestep(p, sh)
    torch.cuda.synchronize()

    # ---- device-timed region: K steps, a CUDA-event pair around every step on its stream ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_begin, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        with torch.cuda.stream(stream):
            t_begin.record(stream)
            for i in range(args.steps):
                p.time_step_seed = args.warmup + i
                ev[i][0].record(stream)
                level.perform_timestep(p, sh)
                ev[i][1].record(stream)
            t_end.record(stream)
        torch.cuda.synchronize()
        # steady-state pass of at least --steady-seconds, so that the clock record holds samples
        # under load even when the K timed steps take milliseconds
        n_steady = max(args.steps, int(args.steady_seconds * 1e3 / max(t_begin.elapsed_time(t_end) / args.steps, 1e-3)))
        s_begin, s_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            s_begin.record(stream)
            for i in range(n_steady):
                p.time_step_seed = args.warmup + args.steps + i
                level.perform_timestep(p, sh)
            s_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    total_ms = t_begin.elapsed_time(t_end)
    steady_ms = s_begin.elapsed_time(s_end)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t = torch.tensor([total_ms, steady_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, steady_ms = float(t[0].item()), float(t[1].item())
    force = level.forces()

    # ---- end-to-end through the public API: per step the step parameters go from pinned host
    # memory into the launch and the FP64 drag comes back to pinned host memory, where the host
    # reads it; double-buffered, as a monitoring loop would run: step i + 1 is enqueued before the
    # host waits for step i's drag ----
    pinned_force = [torch.zeros(3, dtype=torch.float64).pin_memory() for _ in range(2)]
    landed = [torch.cuda.Event() for _ in range(2)]
    drag_seen = []
    e2e_steps = args.steps
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for i in range(e2e_steps):
            p.time_step_seed = args.warmup + args.steps + n_steady + i
            level.perform_timestep(p, sh)
            level.forces_async(pinned_force[i % 2].data_ptr(), sh)
            landed[i % 2].record(stream)
            if i > 0:
                landed[(i - 1) % 2].synchronize()
                drag_seen.append(float(pinned_force[(i - 1) % 2][0]))
        landed[(e2e_steps - 1) % 2].synchronize()
        drag_seen.append(float(pinned_force[(e2e_steps - 1) % 2][0]))
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    assert len(drag_seen) == e2e_steps and all(math.isfinite(v) for v in drag_seen)
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_s = float(te.item())

    if rank == 0:
        peak, peak_kind = measured_peaks()
        sb = STORAGE_BYTES[args.storage]
        alg_bytes = cells * 27 * sb * 2
        avg_ms = statistics.mean(step_ms)
        achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
        value = world * cells * args.steps / (total_ms * 1e-3) / 1e6
        e2e_val = world * cells * e2e_steps / e2e_s / 1e6
        cs = clocks.summary()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.storage, args.nz),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "frac_of_8000": round(achieved / 8000.0, 4),
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "timed_span": "per-step CUDA events around the cumulant launch and the 1-CTA FP64 drag reduction",
                         "traffic": traffic_record(args.storage)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_val, 2), "unit": "MLUPS",
                    "h2d_bytes_per_step": C.sizeof(capi.StepParams), "d2h_bytes_per_step": 24},
            # per step: ghost fill, fast kernel, general kernel (blocks at the sphere), FP64 drag reduction
            "gpu_launches": 4 * args.steps,
            "clocks": cs,
            "steady": {"steps": n_steady, "seconds": round(steady_ms / 1e3, 3),
                       "ms_per_step": round(steady_ms / n_steady, 4),
                       "mlups": round(world * cells * n_steady / (steady_ms * 1e-3) / 1e6, 2),
                       "note": "timed after the K steps under the same clock record"},
            "tuning": tuning,
            "drag_fx_lattice": force[0],
            "cd_after_timed_steps": force[0] * case.meta["drag_scale"],
        }
    extras = rank == 0 and world == 1
    if extras:
        if args.q19_steps > 0:
            from openaerolab_alpha_01_b200.octree import benchmark_periodic_box
            q = [benchmark_periodic_box(256, args.q19_steps, precision=dt) for dt in (np.float32, np.float64)]
            for r in q:
                r["roofline_frac"] = round(r["achieved_gbs"] / peak, 4)
            line["octree_q19"] = q
            from openaerolab_alpha_01_b200.octree import benchmark_naca
            c3 = benchmark_naca(steps=args.q19_steps)
            c3["roofline_frac"] = round(c3["achieved_gbs"] / peak, 4)
            line["octree_config3"] = c3
        if args.kbc_steps > 0:
            from openaerolab_alpha_01_b200.workloads import benchmark_entropic
            kb = benchmark_entropic(128, steps=args.kbc_steps, warmup=3, math="fast")
            kb["roofline_frac"] = round(kb["achieved_gbs"] / peak, 4)
            kb["bound"] = "FP32 issue (13-moment Newton sweeps and entropy evaluations), not HBM"
            ex = benchmark_entropic(128, steps=args.kbc_steps, warmup=3, math="exact")
            kb["exact_math"] = {"mlups": ex["mlups"], "ms_per_step": ex["ms_per_step"],
                                "note": "software exp/log shared with the oracle (bit-identical to it)"}
            kb["speedup_vs_exact"] = round(kb["mlups"] / ex["mlups"], 3)
            line["kbc_d3q39"] = kb
        if args.batch_steps > 0:
            from openaerolab_alpha_01_b200.workloads import config4
            line["batched"] = config4(steps=args.batch_steps, storage=args.storage)
        if args.tgv_steps > 0:
            from openaerolab_alpha_01_b200.validation import taylor_green_64
            line["config1"] = [taylor_green_64(steps=args.tgv_steps, c_wale=cw) for cw in (0.0, 0.2)]
        if args.drag_steps > 0:
            from openaerolab_alpha_01_b200.validation import sphere_drag
            line["drag_check"] = sphere_drag(args.drag_steps, args.drag_avg)
        if args.serve_requests > 0:
            from openaerolab_alpha_01_b200.server import config5
            line["served"] = config5(args.serve_requests, 20.0, args.serve_steps, args.storage,
                                     kbc_share=args.serve_kbc_share)
    if rank == 0:
        print(json.dumps(line), flush=True)

    level.close()
    geom.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
