"""Multi-case workloads: the batched form against the plain per-case loop.

Config 4 (batched): 64 independent periodic D3Q27 cumulant boxes, edge drawn (seeded) from
{32, 48, 64, 96, 128}, Re ~ U[100, 2000], u0 ~ U[0.02, 0.08], a Taylor-Green start with a random
phase, FP16-deviation storage. The batched arm admits every case into one block pool and advances
all of them with one launch per kernel per step (one CUDA graph per advance); the plain arm runs
the cases one after another with one `perform_timestep` call per step (the reference's sequential
case loop, src/main.jl:2184-2238). Both arms time the stepping only (CUDA events, synchronised),
with the same kernels.

    python -m openaerolab_alpha_01_b200.workloads --steps 2000 [--cases 64] [--seed 4]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _capi as capi
from .cases import entropic_taylor_green_case, sphere_channel_case, taylor_green_case
from .solver import Batch, Geometry, Level

SIZES = (32, 48, 64, 96, 128)


def config4_cases(n_cases: int = 64, seed: int = 4):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_cases):
        n = int(rng.choice(SIZES))
        re = float(rng.uniform(100.0, 2000.0))
        u0 = float(rng.uniform(0.02, 0.08))
        phase = (float(rng.uniform(0, n)), float(rng.uniform(0, n)))
        c = taylor_green_case(n, u0=u0, re=re, c_wale=0.0, phase=phase)
        c.name = f"tgv{n}_re{re:.0f}_u{u0:.3f}"
        out.append(c)
    return out


def _cuda_sync():
    import torch
    torch.cuda.synchronize()


def run_batched(cases, steps: int, storage: str = "f16", chunk: int = 100):
    """Advance every case `steps` steps in one batch; returns (seconds, batch, member ids, geometries)."""
    import torch
    geoms = [Geometry(c.dom) for c in cases]
    real = sum(g.blocks()[0] for g in geoms)
    ghost = sum(g.blocks()[1] for g in geoms)
    mask = sum(g.blocks()[2] for g in geoms)
    B = Batch(storage=storage, max_real_blocks=real, max_ghost_blocks=max(ghost, 1), max_mask_blocks=max(mask, 1),
              max_members=len(cases))
    ids = [B.add(g, c.params, c.rho, c.vel) for g, c in zip(geoms, cases)]
    s = torch.cuda.Stream()
    B.advance(min(chunk, steps), s)  # capture + warm-up
    s.synchronize()
    # fresh start: re-admit so the timed run starts from the initial state
    for m in ids:
        B.remove(m)
    ids = [B.add(g, c.params, c.rho, c.vel) for g, c in zip(geoms, cases)]
    # the pool's autotuner (its candidates run from this state, which it restores)
    B.tuning = B.autotune(20)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _cuda_sync()
    e0.record(s)
    left = steps
    while left > 0:
        n = min(chunk, left)
        B.advance(n, s)
        left -= n
    e1.record(s)
    s.synchronize()
    return e0.elapsed_time(e1) / 1e3, B, ids, geoms


def run_plain_loop(cases, steps: int, storage: str = "f16", prefetch_ctas: int = 0, persistent: bool = False):
    """The cases one after another, one step call per step; returns (seconds, final states).
    `prefetch_ctas`, `persistent`: the launch tuning every level uses (the batch's choice, for a
    like-for-like comparison)."""
    import torch
    s = torch.cuda.Stream()
    levels = []
    for c in cases:
        g = Geometry(c.dom)
        L = Level(g, storage=storage)
        L.prefetch_ctas = prefetch_ctas
        L.persistent = persistent
        L.init_equilibrium(c.rho, c.vel)
        L.perform_timestep(c.params, s)  # warm-up of the code path
        L.init_equilibrium(c.rho, c.vel)
        levels.append((g, L))
    _cuda_sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for (g, L), c in zip(levels, cases):
        for _ in range(steps):
            L.perform_timestep(c.params, s)
    e1.record(s)
    s.synchronize()
    return e0.elapsed_time(e1) / 1e3, levels


def config4(steps: int = 2000, n_cases: int = 64, seed: int = 4, storage: str = "f16", check_members: int = 8):
    cases = config4_cases(n_cases, seed)
    cells = sum(c.dom.n_blocks * 512 for c in cases)
    tb, B, ids, geoms = run_batched(cases, steps, storage)
    tp, levels = run_plain_loop(cases, steps, storage, B.tuning["prefetch_ctas"], B.tuning["persistent"])
    # batch invariance on the first members: bit-identical to the plain loop's result
    same = 0
    for i in range(min(check_members, len(cases))):
        fb = B.state(ids[i])[0]
        fp = levels[i][1].state()[0]
        same += int(np.array_equal(fb, fp))
    # accuracy: Taylor-Green kinetic energy against the analytic decay exp(-4 nu k^2 t), FP16 storage
    errs = []
    for i in range(min(check_members, len(cases))):
        c = cases[i]
        _, rho, vel = B.state(ids[i])
        ke = 0.5 * np.sum(rho * (vel ** 2).sum(0))
        ke0 = 0.5 * np.sum(c.rho * (c.vel ** 2).sum(0))
        expect = np.exp(-4 * c.meta["nu"] * c.meta["k"] ** 2 * steps)
        errs.append(abs(ke / ke0 - expect) / expect)
    out = {
        "workload": f"config4_{n_cases}cases_tgv_{steps}steps_{storage}",
        "cases": n_cases, "cells": cells, "steps": steps,
        "batched": {"seconds": round(tb, 4), "cases_per_s": round(n_cases / tb, 3),
                    "mlups": round(cells * steps / tb / 1e6, 1)},
        "plain_loop": {"seconds": round(tp, 4), "cases_per_s": round(n_cases / tp, 3),
                       "mlups": round(cells * steps / tp / 1e6, 1)},
        "speedup": round(tp / tb, 3),
        "tuning": B.tuning,
        "bit_identical_members_checked": f"{same}/{min(check_members, len(cases))}",
        "tgv_ke_rel_error_max": float(max(errs)) if errs else None,
    }
    for g, L in levels:
        L.close(); g.close()
    B.close()
    for g in geoms:
        g.close()
    return out


# algorithmic HBM bytes of one D3Q39 KBC cell update (FP32): populations read + written (2 x 39 x 4)
# and the multiplier cache read + written (2 x 13 x 4); the macro stores and the velocity reads of
# the WALE gradient (28 B) are not counted
KBC_BYTES_PER_CELL = 2 * 39 * 4 + 2 * 13 * 4


def benchmark_entropic(n: int = 128, steps: int = 50, warmup: int = 5, u0: float = 0.1, re: float = 1000.0,
                       math: str = "fast") -> dict:
    """Time `steps` D3Q39 entropic KBC steps of an n^3 periodic Taylor-Green box (one CUDA graph,
    CUDA events on the launching stream). math "fast": CUDA's expf / logf; "exact": the software
    exp / log shared with the oracle."""
    import torch
    case = entropic_taylor_green_case(n, u0=u0, re=re)
    geom = Geometry(case.dom)
    lvl = Level(geom, "entropic", math=math)
    lvl.init_equilibrium(case.rho, case.vel)
    s = torch.cuda.Stream()
    lvl.advance(case.params, warmup, s)
    lvl.advance(case.params, steps, s)  # capture the timed graph outside the timed region
    s.synchronize()
    m0 = lvl.mass_momentum()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    lvl.advance(case.params, steps, s)
    e1.record(s)
    s.synchronize()
    ms = e0.elapsed_time(e1) / steps
    m1 = lvl.mass_momentum()
    cells = n ** 3
    out = {"workload": f"kbc_d3q39_taylor_green_{n}^3_f32_bisection_wale_{math}_math", "cells": cells, "steps": steps,
           "ms_per_step": round(ms, 4), "mlups": round(cells / ms / 1e3, 1), "bytes_per_cell": KBC_BYTES_PER_CELL,
           "achieved_gbs": round(cells * KBC_BYTES_PER_CELL / ms / 1e6, 1),
           "mass_drift_rel": float(abs(m1[0] - m0[0]) / m0[0]), "gpu_launches": steps}
    lvl.close()
    geom.close()
    return out


def benchmark_amr(steps: int = 50, warmup: int = 5, storage: str = "f16", nx: int = 256, ny: int = 128, nz: int = 128,
                  diameter_fine: float = 48.0, re: float = 1000.0, u: float = 0.05) -> dict:
    """Two-level block AMR of the sphere channel: the coarse 256x128x128 channel of config 2 and a
    fine level (2x resolution) over the box [32,128) x [32,96) x [32,96) coarse cells around the
    sphere (diameter 24 coarse = 48 fine cells, centred at x = 64). Half-way walls on both levels,
    the legacy level-viscosity rule (tau_c - 1/2 = 2 (tau_f - 1/2)), Re on the fine diameter. n
    coarse steps per CUDA graph, timed with CUDA events; MLUPS on the work W = coarse cells +
    2 x fine cells per coarse step (src/octree_q19/src/run.jl:99 counts AMR work the same way)."""
    import torch
    from . import _capi as capi
    from .amr import Hierarchy, blocks_in_box, level_taus, refine
    from .solver import apply_analytic_sphere_obstacle, build_box, default_step_params
    coarse = build_box(nx // 8, ny // 8, nz // 8)
    centre = (64.0, ny / 2.0, nz / 2.0)
    apply_analytic_sphere_obstacle(coarse, centre, diameter_fine / 4.0)
    fine = refine(coarse, blocks_in_box(coarse, (32, 32, 32), (128, 96, 96)))
    apply_analytic_sphere_obstacle(fine, tuple(2 * c for c in centre), diameter_fine / 2.0)
    nu_f = u * diameter_fine / re
    taus = level_taus(3.0 * nu_f + 0.5, 2)
    P = [default_step_params(tau=t, c_wale=0.2, u_inlet=u, solid_bc=capi.OAL_SOLID_HALFWAY) for t in taus]
    H = Hierarchy([coarse, fine], storage=storage)
    for lvl, d in enumerate([coarse, fine]):
        n = d.n_blocks * 512
        vel = np.zeros((3, d.n_blocks, 512))
        vel[0] = u
        if d.obstacle is not None:
            vel[0][d.obstacle.astype(bool)] = 0.0
        H.level(lvl).init_equilibrium(np.ones((d.n_blocks, 512)), vel)
    s = torch.cuda.Stream()
    H.advance(P, warmup, s)
    H.advance(P, steps, s)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    H.advance(P, steps, s)
    e1.record(s)
    s.synchronize()
    ms = e0.elapsed_time(e1) / steps
    cells = [coarse.n_blocks * 512, fine.n_blocks * 512]
    work = cells[0] + 2 * cells[1]
    bpc = 2 * 27 * {"f16": 2, "bf16": 2, "f32": 4, "f64": 8}[storage]
    _, rho_f, vel_f = H.level(1).state()
    ok = bool(np.all(np.isfinite(vel_f)))
    H.close()
    return {"workload": f"amr2_sphere_channel_{nx}x{ny}x{nz}_fine_box_96x64x64_{storage}", "coarse_cells": cells[0],
            "fine_cells": cells[1], "work_per_coarse_step": work, "steps": steps, "ms_per_coarse_step": round(ms, 4),
            "mlups": round(work / ms / 1e3, 1), "bytes_per_update": bpc,
            "achieved_gbs": round(work * bpc / ms / 1e6, 1), "finite": ok,
            "gpu_launches_per_coarse_step": "level 0: ghost fill, fast, general; level 1 (x2): parent nodes, interpolation positions, ghost fill, fast, general; restriction; 3 snapshot copies"}


def benchmark_svv(steps: int = 100, warmup: int = 20, storage: str = "f16", eps_yz: float = 0.004,
                  eps_x: float = 0.0) -> dict:
    """Time the config-2 channel (256 x 128 x 128, sphere D 24) with and without the spectral
    vanishing viscosity filter (one CUDA graph of `steps` steps each, CUDA events)."""
    import torch
    case = sphere_channel_case(256, 128, 128, diameter=24.0, centre_x=64.0, u_inlet=0.05, re=1000.0)
    geom = Geometry(case.dom)
    lvl = Level(geom, storage=storage)
    lvl.init_equilibrium(case.rho, case.vel)
    cells = case.dom.n_blocks * 512
    out = {"workload": f"svv_sphere_channel_256x128x128_{storage}_eps_yz{eps_yz:g}_eps_x{eps_x:g}", "cells": cells,
           "steps": steps}
    for name, (ex, eyz) in (("off", (0.0, 0.0)), ("svv", (eps_x, eps_yz))):
        p = capi.StepParams.from_buffer_copy(case.params)
        p.svv_x_epsilon = ex
        p.svv_yz_epsilon = eyz
        lvl.execute_timestep_batch(p, warmup)
        lvl.execute_timestep_batch(p, steps)  # the timed graph, captured outside the timed region
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lvl.execute_timestep_batch(p, steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_step": round(ms, 4), "mlups": round(cells / ms / 1e3, 1)}
    filt = out["svv"]["ms_per_step"] - out["off"]["ms_per_step"]
    bytes_per_cell = 3 * 27 * {"f16": 2, "bf16": 2, "f32": 4, "f64": 8}[storage]
    out["filter_ms"] = round(filt, 4)
    out["filter_gbs"] = round(cells * bytes_per_cell / (filt * 1e-3) / 1e9, 1) if filt > 0 else None
    lvl.close()
    geom.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--storage", default="f16")
    ap.add_argument("--kbc", type=int, default=0,
                    help="instead: time the D3Q39 KBC level on an N^3 periodic Taylor-Green box")
    ap.add_argument("--warmup", type=int, default=5, help="untimed steps before the D3Q39 measurement")
    ap.add_argument("--kbc-math", default="fast", choices=("fast", "exact"),
                    help="D3Q39: CUDA's expf / logf (fast) or the software exp / log shared with the oracle")
    ap.add_argument("--svv", action="store_true",
                    help="instead: time the config-2 channel with and without the SVV filter (y-z, eps 0.004)")
    args = ap.parse_args()
    t0 = time.time()
    if args.svv:
        print(json.dumps(benchmark_svv(steps=args.steps, warmup=args.warmup, storage=args.storage)))
        return
    if args.kbc > 0:
        print(json.dumps(benchmark_entropic(args.kbc, steps=args.steps, warmup=args.warmup, math=args.kbc_math)))
        return
    r = config4(args.steps, args.cases, args.seed, args.storage)
    r["wall_s"] = round(time.time() - t0, 1)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
