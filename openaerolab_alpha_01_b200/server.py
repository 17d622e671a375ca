"""Serving LBM solves: continuous batching over one block pool.

Requests arrive (Poisson, rate lambda); each asks for `steps` steps of a cubic domain, either D3Q27
cumulant — a sphere-in-channel (sphere diameter 0.2 N, inlet u = 0.05, half-way walls with the
FP64 drag) or a periodic Taylor-Green box — or D3Q39 entropic KBC on the same two kinds of domain
(the KBC channel's drag comes from the surface-stress mapping on the sphere's triangles, the
reference's force method for that path). The server keeps every
admitted D3Q27 solve resident in one `Batch`, advanced together in ticks of `tick_steps` steps
(one CUDA graph per tick, one launch per kernel per step for the whole mix), and every admitted
KBC solve resident as its own level on its own stream, advanced in the same ticks so that its
kernels run beside the pool's. Solves that reached their step count retire at the end of a tick,
and arrived requests are admitted whenever the pool (D3Q27) or the KBC share of the HBM budget
has room — requests that arrive while others run join at the next tick. Latency = completion -
arrival, wall clock.

The reference serialises solves (one process per job behind a GPU lock,
apps/airfoil_web/src/gpu_lock.jl:1-11; sequential case queue src/main.jl:2184-2238);
`serve_sequential` is that baseline on the same kernels.

    python -m openaerolab_alpha_01_b200.server --requests 48 --rate 20 --steps 5000
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from .cases import entropic_taylor_green_case, sphere_channel_case, taylor_green_case
from .solver import Batch, Geometry, Level, default_entropic_params, default_surface_params
from .surface import sphere_mesh

# device bytes of one block in a pool (populations x2, rho, velocity x2)
_POP_BYTES = {"f16": 2, "bf16": 2, "f32": 4, "f64": 8}


# device bytes per cell of a D3Q39 KBC level (FP32 populations x2, 13 multipliers, rho, velocity x2)
KBC_BYTES_PER_CELL = 2 * 39 * 4 + 13 * 4 + 4 + 2 * 3 * 4


def block_bytes(storage: str) -> tuple[int, int]:
    """(real, ghost) block cost in a pool."""
    es = _POP_BYTES[storage]
    ms = 8 if storage == "f64" else 4
    return 2 * 27 * 512 * es + 7 * 512 * ms + 27 * 4 + 64, 2 * 27 * 512 * es


@dataclass
class Request:
    rid: int
    arrival: float
    n: int
    kind: str  # "channel" | "box"
    re: float
    steps: int
    u0: float = 0.05
    operator: str = "cumulant"  # "cumulant" (D3Q27) | "entropic" (D3Q39 KBC, periodic boxes)
    # filled by the server
    rejected: bool = False
    admitted: float = math.nan
    done: float = math.nan
    checksum: tuple = ()
    drag: float = math.nan

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def make_requests(n_requests: int = 48, rate: float = 20.0, steps: int = 5000, n_min: int = 32, n_max: int = 192,
                  seed: int = 5, kbc_share: float = 0.0) -> list[Request]:
    """Poisson arrivals; edge log-uniform in [n_min, n_max] rounded to a multiple of 8; half
    channels, half boxes; a fraction `kbc_share` of them D3Q39 KBC, the rest D3Q27."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max))) / 8.0)) * 8
        n = max(n_min, min(n_max, n))
        kind = "channel" if rng.uniform() < 0.5 else "box"
        re = float(math.exp(rng.uniform(math.log(100.0), math.log(5000.0))))
        operator = "cumulant"
        if kbc_share > 0.0 and rng.uniform() < kbc_share:
            operator = "entropic"
        out.append(Request(i, t, n, kind, re, steps, operator=operator))
    return out


def build_case(req: Request):
    if req.operator == "entropic":
        if req.kind == "channel":
            case = sphere_channel_case(req.n, req.n, req.n, diameter=0.2 * req.n, centre_x=req.n / 4.0,
                                       u_inlet=req.u0, re=req.re)
            case.params = default_entropic_params(tau=float(case.params.tau), c_wale=0.2, u_inlet=req.u0)
            return case
        return entropic_taylor_green_case(req.n, u0=req.u0, re=req.re, c_wale=0.2)
    if req.kind == "channel":
        return sphere_channel_case(req.n, req.n, req.n, diameter=0.2 * req.n, centre_x=req.n / 4.0,
                                   u_inlet=req.u0, re=req.re)
    return taylor_green_case(req.n, u0=req.u0, re=req.re, c_wale=0.2)


def kbc_drag(req: Request, case, L: Level) -> np.ndarray:
    """The force on a D3Q39 channel's sphere by the surface-stress mapping, the reference's force
    method for the entropic path (compute_aerodynamics!, src/forces/surface.jl:1577-1660): the
    sphere's triangles attached to the level and its stresses integrated in FP64 (lattice units).
    Periodic boxes have no body: zeros."""
    if req.kind != "channel":
        return np.zeros(3)
    m = case.meta
    L.set_surface(sphere_mesh(m["centre"], m["diameter"] / 2.0))
    return L.surface_forces(default_surface_params(tau=float(case.params.tau), c_wale=float(case.params.c_wale)))["total"]


def _finish(req: Request, totals: np.ndarray, drag: np.ndarray, t: float):
    """A solve's result: its FP64 drag and FP64 mass/momentum totals (computed on the GPU)."""
    req.done = t
    req.checksum = tuple(float(v) for v in totals) + tuple(float(v) for v in drag)
    req.drag = float(drag[0])


def serve(requests: list[Request], budget_bytes: float = 150e9, storage: str = "f16", tick_steps: int = 250,
          max_members: int = 256, keep_states: bool = False, max_active_cells: int = 12_000_000,
          kbc_budget_share: float = 0.25, max_active_kbc_cells: int = 4_000_000):
    """Continuous batching in real time. Returns a summary and fills the requests' timestamps.

    `max_active_cells` bounds the resident D3Q27 work: a few million cells already fill a B200,
    so admitting more only makes every resident solve slower (all of them finish late); with the
    bound, solves finish in arrival order while the GPU stays full. KBC solves (about fifty
    times the arithmetic per cell update) have their own bound `max_active_kbc_cells` and draw
    their levels from `kbc_budget_share` of the HBM budget; the D3Q27 pool gets the rest."""
    import torch
    rb, gb = block_bytes(storage)
    has_kbc = any(r.operator == "entropic" for r in requests)
    kbc_budget = budget_bytes * kbc_budget_share if has_kbc else 0.0
    pool_budget = budget_bytes - kbc_budget
    # the pool: its budget split 60:40 between real and ghost blocks (small cubes carry many ghost
    # blocks per real one), bounded by the 2^32-element population index of a pool
    max_blocks = (1 << 32) // (27 * 512) - 1
    real = int(min(pool_budget * 0.6 / rb, max_blocks * 0.6))
    ghost = int(min(pool_budget * 0.4 / gb, max_blocks * 0.4))
    B = Batch(storage=storage, max_real_blocks=real, max_ghost_blocks=ghost, max_mask_blocks=max(real // 16, 64),
              max_members=max_members)
    pool_stream = torch.cuda.Stream()
    pending = sorted(requests, key=lambda r: r.arrival)
    active: dict[int, tuple[Request, Geometry, int]] = {}  # member -> (request, geometry, steps done)
    kbc: dict[int, list] = {}  # rid -> [request, geometry, level, params, stream, steps done]
    kbc_bytes = 0.0
    states = {}
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    finished = 0
    ticks = 0
    prepared = {}  # rid -> case built on the host while the GPU runs a tick

    def admit(req: Request) -> str:
        """'ok', 'wait' (no room now) or 'never' (larger than its whole share)."""
        nonlocal kbc_bytes
        case = prepared.pop(req.rid, None) or build_case(req)
        if req.operator == "entropic":
            need = req.n ** 3 * KBC_BYTES_PER_CELL
            if need > kbc_budget:
                return "never"
            cells = sum(e[0].n ** 3 for e in kbc.values())
            if kbc and (kbc_bytes + need > kbc_budget or cells + req.n ** 3 > max_active_kbc_cells):
                prepared[req.rid] = case
                return "wait"
            g = Geometry(case.dom)
            L = Level(g, "entropic")
            L.init_equilibrium(case.rho, case.vel)
            kbc[req.rid] = [req, g, L, case.params, torch.cuda.Stream(), 0, case]
            kbc_bytes += need
            return "ok"
        if active and sum(r.n ** 3 for r, _, _ in active.values()) + req.n ** 3 > max_active_cells:
            prepared[req.rid] = case
            return "wait"
        g = Geometry(case.dom)
        m = B.try_add(g, case.params, case.rho, case.vel)
        if m is None:
            g.close()
            if not active:
                return "never"  # larger than the whole pool: it can never be admitted
            prepared[req.rid] = case
            return "wait"
        active[m] = (req, g, 0)
        return "ok"

    while finished < len(requests):
        # admit arrived requests in arrival order; a request that must wait holds back the later
        # ones of its operator only
        blocked = set()
        for req in list(pending):
            if req.arrival > now():
                break
            if req.operator in blocked:
                continue
            verdict = admit(req)
            if verdict == "wait":
                blocked.add(req.operator)
                continue
            pending.remove(req)
            if verdict == "never":
                req.rejected = True
                finished += 1
            else:
                req.admitted = now()
        if not active and not kbc:
            if pending:
                time.sleep(max(0.0, pending[0].arrival - now()))
            continue
        # one tick: every resident solve advances by the same number of steps (the smallest
        # remaining count bounds it); the pool and each KBC level on their own streams
        left = [req.steps - done for req, _, done in active.values()] + [e[0].steps - e[5] for e in kbc.values()]
        n = min(tick_steps, min(left))
        if active:
            B.advance(n, stream=pool_stream)
        for e in kbc.values():
            e[2].execute_timestep_batch(e[3], n, stream=e[4])
        ticks += 1
        # host work overlapping the tick: build the cases of requests that have arrived
        for req in pending:
            if req.arrival > now():
                break
            if req.rid not in prepared:
                prepared[req.rid] = build_case(req)
        torch.cuda.synchronize()
        for m in list(active):
            req, g, done = active[m]
            done += n
            active[m] = (req, g, done)
            if done >= req.steps:
                _finish(req, B.mass_momentum(m), B.forces(m), now())
                if keep_states:
                    states[req.rid] = B.state(m)[0]
                B.remove(m)
                g.close()
                del active[m]
                finished += 1
        for rid in list(kbc):
            e = kbc[rid]
            e[5] += n
            if e[5] >= e[0].steps:
                req, g, L = e[0], e[1], e[2]
                _finish(req, L.mass_momentum(), kbc_drag(req, e[6], L), now())
                if keep_states:
                    states[req.rid] = L.state()[0]
                L.close()
                g.close()
                kbc_bytes -= req.n ** 3 * KBC_BYTES_PER_CELL
                del kbc[rid]
                finished += 1
    makespan = now()
    B.close()
    return summarize(requests, makespan, "served", ticks=ticks, max_active_cells=max_active_cells), states


def serve_sequential(requests: list[Request], storage: str = "f16", keep_states: bool = False):
    """The baseline: one solve at a time in arrival order (each as its own level, CUDA graph per
    solve; KBC solves as FP32 entropic levels)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    states = {}
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for req in pending:
        if req.arrival > now():
            time.sleep(req.arrival - now())
        case = build_case(req)
        g = Geometry(case.dom)
        L = Level(g, "entropic") if req.operator == "entropic" else Level(g, storage=storage)
        L.init_equilibrium(case.rho, case.vel)
        req.admitted = now()
        left = req.steps
        while left > 0:
            n = min(1000, left)
            L.execute_timestep_batch(case.params, n)
            left -= n
        _finish(req, L.mass_momentum(), kbc_drag(req, case, L) if req.operator == "entropic" else L.forces(), now())
        if keep_states:
            states[req.rid] = L.state()[0]
        L.close()
        g.close()
    return summarize(requests, now(), "sequential"), states


def summarize(requests: list[Request], makespan: float, mode: str, **extra) -> dict:
    done = [r for r in requests if not r.rejected]
    lat = np.array([r.latency for r in done]) if done else np.array([math.nan])
    cells = sum(r.n ** 3 * r.steps for r in done)
    n_kbc = sum(r.operator == "entropic" for r in done)
    return {"mode": mode, "requests": len(requests), "completed": len(done), "completed_d3q39": n_kbc,
            "rejected": len(requests) - len(done),
            "makespan_s": round(makespan, 3), "cases_per_s": round(len(done) / makespan, 3),
            "latency_p50_s": round(float(np.percentile(lat, 50)), 3),
            "latency_p99_s": round(float(np.percentile(lat, 99)), 3),
            "mlups": round(cells / makespan / 1e6, 1), **extra}


def config5(n_requests: int = 48, rate: float = 20.0, steps: int = 5000, storage: str = "f16", seed: int = 5,
            budget_bytes: float = 150e9, kbc_share: float = 0.5):
    reqs = make_requests(n_requests, rate, steps, seed=seed, kbc_share=kbc_share)
    served, _ = serve(reqs, budget_bytes=budget_bytes, storage=storage)
    served_cs = {r.rid: r.checksum for r in reqs}
    reqs2 = make_requests(n_requests, rate, steps, seed=seed, kbc_share=kbc_share)
    seq, _ = serve_sequential(reqs2, storage=storage)
    same = sum(int(served_cs[r.rid] == r.checksum) for r in reqs2)
    mix = "d3q27only" if kbc_share <= 0 else f"d3q39share{kbc_share:g}"
    return {"workload": f"config5_{n_requests}req_rate{rate:g}_{steps}steps_{storage}_{mix}",
            "served": served, "sequential": seq,
            "cases_per_s_ratio": round(served["cases_per_s"] / seq["cases_per_s"], 3),
            "identical_results": f"{same}/{n_requests}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--storage", default="f16")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--kbc-share", type=float, default=0.5, help="fraction of D3Q39 KBC requests")
    args = ap.parse_args()
    print(json.dumps(config5(args.requests, args.rate, args.steps, args.storage, args.seed, args.budget_gb * 1e9,
                             args.kbc_share)))


if __name__ == "__main__":
    main()
