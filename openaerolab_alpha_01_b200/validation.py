"""Accuracy runs of the two uniform-grid D3Q27 workloads, on the GPU through the level API.

* ``taylor_green_64`` — the 64^3 fully periodic Taylor-Green vortex in FP64 storage and arithmetic
  (u0 = 0.05, Re = 100 with L = 64 / (2 pi), 1000 steps). It reports the kinetic-energy ratio
  against the analytic decay exp(-4 nu k^2 t), measured both from t = 0 and, in the form of the
  reference's gate (tools/tests/q19_octree_step.jl:85-107), from t = steps / 5 on, and the L2
  error of the velocity field against the analytic field u0 exp(-2 nu k^2 t) (sin kx cos ky,
  -cos kx sin ky, 0).
* ``sphere_drag`` — the 256 x 128 x 128 sphere channel (D = 24 at x = 64, inlet u = 0.05 at
  src/collision/kernel_cumulant.jl:235-239, zero-gradient outlet :240-245, lateral mirrors,
  Re = 1000, WALE c_w = 0.2, half-way bounce-back with the FP64 momentum-exchange force of
  src/octree_q19/src/stream.jl:248-256 on the 27 links) run once per population storage (FP64,
  FP32, FP16 and BF16 deviations; FP32 arithmetic for all but FP64; the 16-bit storages with
  stochastic rounding, the default, and with rounding to nearest, ``f16:rn``). The drag of every
  step is copied to pinned host memory in stream order. Reported per storage: the drag
  coefficient averaged over the last ``avg_last`` steps and its relative difference from FP64,
  and the same over the deterministic window [1000, 7000) of the start-up, before the wake
  breaks its mirror symmetry. At Re = 1000 the symmetric wake is unstable: runs whose rounding
  differs leave it at different times (FP32 near 14,000 steps, FP64 after 20,000), so a
  time average over a late window compares different wake states rather than precisions.

    python -m openaerolab_alpha_01_b200.validation [--drag-steps 20000] [--avg-last 5000]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .cases import sphere_channel_case, taylor_green_case
from .solver import Geometry, Level, kinetic_energy


def taylor_green_fields_at(case, t: float):
    """Analytic velocity of the decaying 2-D Taylor-Green vortex of ``case`` at step t."""
    d = case.dom
    gx, gy, _ = d.cell_positions()
    k = case.meta["k"]
    amp = case.meta["u0"] * np.exp(-2.0 * case.meta["nu"] * k * k * t)
    x, y = gx - 0.5, gy - 0.5
    u = np.zeros((3,) + gx.shape)
    u[0] = amp * np.sin(k * x) * np.cos(k * y)
    u[1] = -amp * np.cos(k * x) * np.sin(k * y)
    return u


def taylor_green_64(n: int = 64, steps: int = 1000, c_wale: float = 0.0, storage: str = "f64",
                    u0: float = 0.05, re: float = 100.0, device: int = 0) -> dict:
    """Config 1 on the GPU: KE decay and L2 velocity error of the periodic Taylor-Green box."""
    import torch
    case = taylor_green_case(n, u0=u0, re=re, c_wale=c_wale)
    g = Geometry(case.dom, device=device)
    L = Level(g, storage=storage)
    L.init_equilibrium(case.rho, case.vel)
    s = torch.cuda.Stream(device=device)
    s1 = steps // 5
    ke0 = kinetic_energy(case.rho, case.vel)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    L.advance(case.params, s1, s)
    s.synchronize()
    _, rho1, vel1 = L.state()
    ke1 = kinetic_energy(rho1, vel1)
    L.advance(case.params, steps - s1, s)
    e1.record(s)
    s.synchronize()
    ms = e0.elapsed_time(e1)
    _, rho2, vel2 = L.state()
    ke2 = kinetic_energy(rho2, vel2)
    nu, k = case.meta["nu"], case.meta["k"]
    expect_full = float(np.exp(-4.0 * nu * k * k * steps))
    expect_gate = float(np.exp(-4.0 * nu * k * k * (steps - s1)))
    ua = taylor_green_fields_at(case, steps)
    l2 = float(np.sqrt(np.sum((vel2 - ua) ** 2) / np.sum(ua ** 2)))
    mm = L.mass_momentum()
    L.close()
    g.close()
    return {
        "workload": f"taylor_green_{n}^3_periodic_{storage}_u{u0}_re{re:g}_cwale{c_wale:g}",
        "steps": steps, "nu": nu, "tau": case.meta["tau"],
        "ke_ratio": ke2 / ke0, "ke_expected": expect_full, "ke_rel_error": abs(ke2 / ke0 - expect_full) / expect_full,
        "ke_ratio_from_s1": ke2 / ke1, "ke_expected_from_s1": expect_gate,
        "ke_rel_error_from_s1": abs(ke2 / ke1 - expect_gate) / expect_gate,
        "l2_velocity_error": l2, "mass": float(mm[0]), "finite": bool(np.all(np.isfinite(vel2))),
        "gpu_ms_total": round(ms, 3), "mlups": round(n ** 3 * steps / ms / 1e3, 1),
    }


def sphere_drag_run(storage: str, steps: int, nx: int = 256, ny: int = 128, nz: int = 128, diameter: float = 24.0,
                    centre_x: float = 64.0, device: int = 0) -> dict:
    """One storage of the config-2 accuracy run: per-step FP64 drag and lift coefficients.
    `storage` is a storage name, with ":rn" for rounding to nearest (16-bit storages)."""
    import torch
    name, _, mode = storage.partition(":")
    case = sphere_channel_case(nx, ny, nz, diameter=diameter, centre_x=centre_x)
    g = Geometry(case.dom, device=device)
    L = Level(g, storage=name, rounding="nearest" if mode == "rn" else "stochastic")
    L.init_equilibrium(case.rho, case.vel)
    p = case.params
    s = torch.cuda.Stream(device=device)
    forces = torch.zeros((steps, 3), dtype=torch.float64).pin_memory()
    base = forces.data_ptr()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record(s)
    for i in range(steps):
        p.time_step_seed = i
        L.perform_timestep(p, s)
        L.forces_async(base + 24 * i, s)
    e1.record(s)
    s.synchronize()
    ms = e0.elapsed_time(e1)
    F = forces.numpy().copy()
    _, rho, vel = L.state()
    finite = bool(np.all(np.isfinite(vel)))
    L.close()
    g.close()
    scale = case.meta["drag_scale"]
    return {"storage": storage, "cd": F[:, 0] * scale, "cl_y": F[:, 1] * scale, "cl_z": F[:, 2] * scale,
            "finite": finite, "ms_per_step": ms / steps}


DETERMINISTIC_WINDOW = (1000, 7000)


def sphere_drag(steps: int = 20000, avg_last: int = 5000, storages=("f64", "f32", "f16", "bf16", "f16:rn", "bf16:rn"),
                nx: int = 256, ny: int = 128, nz: int = 128, device: int = 0, series_every: int = 0) -> dict:
    """Config 2 accuracy: time-averaged drag coefficient per storage and its difference from FP64."""
    avg_last = min(avg_last, steps)
    runs = {}
    for st in storages:
        runs[st] = sphere_drag_run(st, steps, nx, ny, nz, device=device)
    ref = runs.get("f64")
    out = {"workload": f"sphere_channel_{nx}x{ny}x{nz}_D24_Re1000_cwale0.2_halfway", "steps": steps,
           "average_over_last": avg_last, "storages": {}}
    cd_ref = float(np.mean(ref["cd"][-avg_last:])) if ref else None
    w0, w1 = DETERMINISTIC_WINDOW
    win = steps >= w1
    cdw_ref = float(np.mean(ref["cd"][w0:w1])) if ref is not None and win else None
    out["deterministic_window"] = list(DETERMINISTIC_WINDOW) if win else None
    for st, r in runs.items():
        cd = float(np.mean(r["cd"][-avg_last:]))
        d = {"cd_mean": cd, "cd_std": float(np.std(r["cd"][-avg_last:])),
             "cl_y_mean": float(np.mean(r["cl_y"][-avg_last:])), "cl_z_mean": float(np.mean(r["cl_z"][-avg_last:])),
             "ms_per_step": round(r["ms_per_step"], 4), "finite": r["finite"]}
        bad = np.flatnonzero(~np.isfinite(r["cd"]))
        d["first_nonfinite_step"] = int(bad[0]) + 1 if bad.size else None
        if win:
            d["cd_window_mean"] = float(np.mean(r["cd"][w0:w1]))
        if ref is not None and st != "f64":
            d["cd_rel_diff_vs_f64"] = abs(cd - cd_ref) / abs(cd_ref)
            if win:
                d["cd_window_rel_diff_vs_f64"] = abs(d["cd_window_mean"] - cdw_ref) / abs(cdw_ref)
                d["cd_window_max_rel_diff_vs_f64"] = float(np.max(np.abs(r["cd"][w0:w1] - ref["cd"][w0:w1]) / np.abs(ref["cd"][w0:w1])))
        if series_every:
            d["cd_series"] = [round(float(v), 6) for v in r["cd"][::series_every]]
        out["storages"][st] = d
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--drag-steps", type=int, default=20000)
    ap.add_argument("--avg-last", type=int, default=5000)
    ap.add_argument("--tgv-steps", type=int, default=1000)
    ap.add_argument("--series-every", type=int, default=0)
    args = ap.parse_args()
    t0 = time.time()
    res = {"config1": [taylor_green_64(steps=args.tgv_steps, c_wale=cw) for cw in (0.0, 0.2)]}
    if args.drag_steps > 0:
        res["config2_drag"] = sphere_drag(args.drag_steps, args.avg_last, series_every=args.series_every)
    res["wall_s"] = round(time.time() - t0, 1)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
