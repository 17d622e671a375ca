"""Serving LBM solves: continuous batching over one block pool.

Requests arrive (Poisson, rate lambda); each asks for `steps` steps of a cubic D3Q27 cumulant
domain: a sphere-in-channel (sphere diameter 0.2 N, inlet u = 0.05, half-way walls with the FP64
drag) or a periodic Taylor-Green box. The server keeps every admitted solve resident in one
`Batch`, advances all of them together in ticks of `tick_steps` steps (one CUDA graph per tick,
one launch per kernel per step for the whole mix), retires solves that reached their step count,
and admits arrived requests whenever the pool (the HBM budget) has room — requests that arrive
while others run join at the next tick. Latency = completion - arrival, wall clock.

The reference serialises solves (one process per job behind a GPU lock,
apps/airfoil_web/src/gpu_lock.jl:1-11; sequential case queue src/main.jl:2184-2238);
`serve_sequential` is that baseline on the same kernels.

The served mix of the workload description also contains D3Q39 entropic KBC solves; that
operator has no kernel in this build, so every request here is D3Q27 cumulant.

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
from .cases import sphere_channel_case, taylor_green_case
from .solver import Batch, Geometry, Level

# device bytes of one block in a pool (populations x2, rho, velocity x2)
_POP_BYTES = {"f16": 2, "bf16": 2, "f32": 4, "f64": 8}


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
                  seed: int = 5) -> list[Request]:
    """Poisson arrivals; edge log-uniform in [n_min, n_max] rounded to a multiple of 8; half channels."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max))) / 8.0)) * 8
        n = max(n_min, min(n_max, n))
        kind = "channel" if rng.uniform() < 0.5 else "box"
        re = float(math.exp(rng.uniform(math.log(100.0), math.log(5000.0))))
        out.append(Request(i, t, n, kind, re, steps))
    return out


def build_case(req: Request):
    if req.kind == "channel":
        return sphere_channel_case(req.n, req.n, req.n, diameter=0.2 * req.n, centre_x=req.n / 4.0,
                                   u_inlet=req.u0, re=req.re)
    return taylor_green_case(req.n, u0=req.u0, re=req.re, c_wale=0.2)


def _finish(req: Request, totals: np.ndarray, drag: np.ndarray, t: float):
    """A solve's result: its FP64 drag and FP64 mass/momentum totals (computed on the GPU)."""
    req.done = t
    req.checksum = tuple(float(v) for v in totals) + tuple(float(v) for v in drag)
    req.drag = float(drag[0])


def serve(requests: list[Request], budget_bytes: float = 150e9, storage: str = "f16", tick_steps: int = 250,
          max_members: int = 256, keep_states: bool = False, max_active_cells: int = 12_000_000):
    """Continuous batching in real time. Returns a summary and fills the requests' timestamps.

    `max_active_cells` bounds the resident work: a few million cells already fill a B200, so
    admitting more only makes every resident solve slower (all of them finish late); with the
    bound, solves finish in arrival order while the GPU stays full."""
    rb, gb = block_bytes(storage)
    # the pool: the budget split 60:40 between real and ghost blocks (small cubes carry many ghost
    # blocks per real one), bounded by the 2^32-element population index of a pool
    max_blocks = (1 << 32) // (27 * 512) - 1
    real = int(min(budget_bytes * 0.6 / rb, max_blocks * 0.6))
    ghost = int(min(budget_bytes * 0.4 / gb, max_blocks * 0.4))
    B = Batch(storage=storage, max_real_blocks=real, max_ghost_blocks=ghost, max_mask_blocks=max(real // 16, 64),
              max_members=max_members)
    pending = sorted(requests, key=lambda r: r.arrival)
    active: dict[int, tuple[Request, Geometry, int]] = {}  # member -> (request, geometry, steps done)
    states = {}
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    finished = 0
    ticks = 0
    prepared = {}  # rid -> case built on the host while the GPU runs a tick
    while finished < len(requests):
        # admit every arrived request the pool can hold (in arrival order)
        while pending and pending[0].arrival <= now():
            req = pending[0]
            if active and sum(r.n ** 3 for r, _, _ in active.values()) + req.n ** 3 > max_active_cells:
                break
            case = prepared.pop(req.rid, None) or build_case(req)
            g = Geometry(case.dom)
            m = B.try_add(g, case.params, case.rho, case.vel)
            if m is None:
                g.close()
                prepared[req.rid] = case
                if not active:
                    # larger than the whole pool: it can never be admitted
                    pending.pop(0)
                    req.rejected = True
                    finished += 1
                    continue
                break
            pending.pop(0)
            req.admitted = now()
            active[m] = (req, g, 0)
        if not active:
            if pending:
                time.sleep(max(0.0, pending[0].arrival - now()))
            continue
        # one tick: every resident solve advances together (smallest remaining first bounds the tick)
        n = min(tick_steps, min(req.steps - done for req, _, done in active.values()))
        B.advance(n)
        ticks += 1
        # host work overlapping the tick: build the cases of requests that have arrived
        for req in pending:
            if req.arrival > now():
                break
            if req.rid not in prepared:
                prepared[req.rid] = build_case(req)
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
    makespan = now()
    B.close()
    return summarize(requests, makespan, "served", ticks=ticks, max_active_cells=max_active_cells), states


def serve_sequential(requests: list[Request], storage: str = "f16", keep_states: bool = False):
    """The baseline: one solve at a time in arrival order (each as its own level, CUDA graph per solve)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    states = {}
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for req in pending:
        if req.arrival > now():
            time.sleep(req.arrival - now())
        case = build_case(req)
        g = Geometry(case.dom)
        L = Level(g, storage=storage)
        L.init_equilibrium(case.rho, case.vel)
        req.admitted = now()
        left = req.steps
        while left > 0:
            n = min(1000, left)
            L.execute_timestep_batch(case.params, n)
            left -= n
        _finish(req, L.mass_momentum(), L.forces(), now())
        if keep_states:
            states[req.rid] = L.state()[0]
        L.close()
        g.close()
    return summarize(requests, now(), "sequential"), states


def summarize(requests: list[Request], makespan: float, mode: str, **extra) -> dict:
    done = [r for r in requests if not r.rejected]
    lat = np.array([r.latency for r in done]) if done else np.array([math.nan])
    cells = sum(r.n ** 3 * r.steps for r in done)
    return {"mode": mode, "requests": len(requests), "completed": len(done), "rejected": len(requests) - len(done),
            "makespan_s": round(makespan, 3), "cases_per_s": round(len(done) / makespan, 3),
            "latency_p50_s": round(float(np.percentile(lat, 50)), 3),
            "latency_p99_s": round(float(np.percentile(lat, 99)), 3),
            "mlups": round(cells / makespan / 1e6, 1), **extra}


def config5(n_requests: int = 48, rate: float = 20.0, steps: int = 5000, storage: str = "f16", seed: int = 5,
            budget_bytes: float = 150e9):
    reqs = make_requests(n_requests, rate, steps, seed=seed)
    served, _ = serve(reqs, budget_bytes=budget_bytes, storage=storage)
    served_cs = {r.rid: r.checksum for r in reqs}
    reqs2 = make_requests(n_requests, rate, steps, seed=seed)
    seq, _ = serve_sequential(reqs2, storage=storage)
    same = sum(int(served_cs[r.rid] == r.checksum) for r in reqs2)
    return {"workload": f"config5_{n_requests}req_rate{rate:g}_{steps}steps_{storage}_d3q27only",
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
    args = ap.parse_args()
    print(json.dumps(config5(args.requests, args.rate, args.steps, args.storage, args.seed, args.budget_gb * 1e9)))


if __name__ == "__main__":
    main()
