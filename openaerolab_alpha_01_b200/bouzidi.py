"""Boundary cells and link fractions of the linear Bouzidi wall on a D3Q27 level.

The reference builds them on the host once per level (compute_bouzidi_qmap_sparse,
src/geometry/bouzidi_setup.jl:175-390): for every fluid cell, every link k whose ray from the
cell centre hits the body within one link (0 < q <= 1) and whose neighbour x + c_k is solid is
kept, q stored as Float16; a cell with at least one kept link is a boundary cell. This module
does the same for the analytic sphere (q_geometry "sphere_analytic", compute_q_for_sphere_cell
and ray_sphere_first_hit, src/geometry/bouzidi_math.jl:127-205), in Float64, vectorised over the
cells; the result feeds solver.Level.set_bouzidi. Cell centres sit at (global index - 0.5) dx.
"""
from __future__ import annotations

import numpy as np

from .solver import BlockDomain

_K = np.arange(27)
CX, CY, CZ = _K % 3 - 1, (_K // 3) % 3 - 1, _K // 9 - 1


def ray_sphere_first_hit(origin: np.ndarray, dir_unit: np.ndarray, centre, radius: float) -> np.ndarray:
    """Distance along dir_unit to the first crossing of the sphere ahead of each origin (inf = none).
    origin (..., 3), dir_unit (3,)."""
    oc = origin - np.asarray(centre, np.float64)
    b = oc @ dir_unit
    c = np.einsum("...i,...i->...", oc, oc) - radius * radius
    disc = b * b - c
    with np.errstate(invalid="ignore"):
        s = np.sqrt(disc)
    t1, t2 = -b - s, -b + s
    eps = 1.0e-10 * max(radius, 1.0)
    t = np.where(t1 > eps, t1, np.where(t2 > eps, t2, np.inf))
    return np.where(disc < 0.0, np.inf, t)


def sphere_qmap(dom: BlockDomain, centre, radius: float, dx: float = 1.0):
    """Boundary cells (n, 4) int32 (block, x, y, z), 1-based, in block then z, y, x order, and
    their q (n, 27) float16 (0 = no wall link). The domain's obstacle mask decides which links are
    kept (the neighbour across the link must be solid)."""
    if dom.obstacle is None:
        raise ValueError("the q map keeps links into solid cells: the domain needs an obstacle mask")
    nb = dom.n_blocks
    solid = dom.obstacle.reshape(nb, 512) != 0
    cell = np.arange(512)
    lx, ly, lz = cell & 7, (cell >> 3) & 7, cell >> 6
    gx, gy, gz = dom.cell_positions()
    pos = np.stack([(gx - 0.5) * dx, (gy - 0.5) * dx, (gz - 0.5) * dx], axis=-1)  # (nb, 512, 3)
    nbr = dom.neighbor_table  # (27, nb), 1-based, 0 = none
    q = np.zeros((nb, 512, 27), np.float64)
    blocks = np.arange(nb)[:, None]
    for k in range(27):
        if k == 13:
            continue
        nx, ny, nz = lx + CX[k], ly + CY[k], lz + CZ[k]
        d = (nx // 8 + 1) + 3 * (ny // 8 + 1) + 9 * (nz // 8 + 1)  # neighbour-block direction per cell
        nbb = nbr[d[None, :], blocks]  # (nb, 512)
        ncell = (nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6)
        nsolid = (nbb > 0) & solid[np.maximum(nbb - 1, 0), np.broadcast_to(ncell, (nb, 512))]
        cand = nsolid & ~solid
        if not cand.any():
            continue
        c = np.array([CX[k], CY[k], CZ[k]], np.float64)
        cmag = float(np.linalg.norm(c))
        t = ray_sphere_first_hit(pos[cand], c / cmag, centre, radius)
        qk = t / (dx * cmag)
        ok = np.isfinite(qk) & (qk > 0.0) & (qk <= 1.0)
        vals = np.where(ok, qk, 0.0)
        q[cand, k] = vals
    has = (q > 0.0).any(axis=2)
    bi, ci = np.nonzero(has)
    cells = np.stack([bi + 1, (ci & 7) + 1, ((ci >> 3) & 7) + 1, (ci >> 6) + 1], axis=1).astype(np.int32)
    return cells, q[bi, ci].astype(np.float16)


def ray_triangle_hits(origin: np.ndarray, dir_unit: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """Two-sided Moller-Trumbore distances (ray_triangle_intersection, bouzidi_math.jl:9-50) of
    every origin (m, 3) along dir_unit (3,) to every triangle (t, 3, 3): (m, t), inf = no hit.
    |det| < 1e-9 misses, the barycentric test admits 64 eps of round-off on the edges, and only
    hits at t > 1e-9 count."""
    eps, bary = 1.0e-9, 64 * np.finfo(np.float64).eps
    v1 = tris[:, 0]
    e1, e2 = tris[:, 1] - v1, tris[:, 2] - v1
    h = np.cross(dir_unit, e2)                       # (t, 3)
    a = np.einsum("ti,ti->t", e1, h)
    ok_a = np.abs(a) >= eps
    f = np.where(ok_a, 1.0 / np.where(ok_a, a, 1.0), 0.0)
    s = origin[:, None, :] - v1[None, :, :]          # (m, t, 3)
    u = f[None, :] * np.einsum("mti,ti->mt", s, h)
    qv = np.cross(s, e1[None, :, :])
    v = f[None, :] * (qv @ dir_unit)
    t = f[None, :] * np.einsum("mti,ti->mt", qv, e2)
    hit = (ok_a[None, :] & (u >= -bary) & (u <= 1.0 + bary) & (v >= -bary) & (u + v <= 1.0 + bary) & (t > eps))
    return np.where(hit, t, np.inf)


def stl_qmap(dom: BlockDomain, triangles, mesh_offset=(0.0, 0.0, 0.0), dx: float = 1.0):
    """Boundary cells, q (float16) and the 1-based triangle of each kept link for a triangle mesh
    (q_geometry "stl_ray": compute_q_for_cell, bouzidi_math.jl:57-125, over the triangles near each
    block, build_block_triangle_map_for_bouzidi, bouzidi_setup.jl:12-58). triangles (T, 3, 3) in
    mesh coordinates; mesh_offset is added to every vertex. Returns (cells (n, 4) int32, q (n, 27)
    float16, tri (n, 27) int32, 0 = none)."""
    if dom.obstacle is None:
        raise ValueError("the q map keeps links into solid cells: the domain needs an obstacle mask")
    tris = np.asarray(triangles, np.float64).reshape(-1, 3, 3) + np.asarray(mesh_offset, np.float64)
    nb = dom.n_blocks
    solid = dom.obstacle.reshape(nb, 512) != 0
    margin = dx * (np.sqrt(3.0) + 1.0)                # max |c| of D3Q27 plus one cell
    bmin = np.floor((tris.min(axis=1) - margin) / (8 * dx)).astype(np.int64) + 1
    bmax = np.floor((tris.max(axis=1) + margin) / (8 * dx)).astype(np.int64) + 1
    cell = np.arange(512)
    lx, ly, lz = cell & 7, (cell >> 3) & 7, cell >> 6
    nbr = dom.neighbor_table
    q = np.zeros((nb, 512, 27), np.float64)
    tri_of = np.zeros((nb, 512, 27), np.int32)
    for b in range(nb):
        bc = dom.coords[b].astype(np.int64)
        near = np.nonzero(np.all((bmin <= bc) & (bc <= bmax), axis=1))[0]
        if near.size == 0:
            continue
        centre = np.stack([((bc[0] - 1) * 8 + lx + 0.5) * dx, ((bc[1] - 1) * 8 + ly + 0.5) * dx,
                           ((bc[2] - 1) * 8 + lz + 0.5) * dx], axis=1)
        for k in range(27):
            if k == 13:
                continue
            nx, ny, nz = lx + CX[k], ly + CY[k], lz + CZ[k]
            d = (nx // 8 + 1) + 3 * (ny // 8 + 1) + 9 * (nz // 8 + 1)
            nbb = nbr[d, b]
            ncell = (nx & 7) | ((ny & 7) << 3) | ((nz & 7) << 6)
            cand = np.nonzero((nbb > 0) & solid[np.maximum(nbb - 1, 0), ncell] & ~solid[b])[0]
            if cand.size == 0:
                continue
            c = np.array([CX[k], CY[k], CZ[k]], np.float64)
            cmag = float(np.linalg.norm(c))
            t = ray_triangle_hits(centre[cand], c / cmag, tris[near])
            j = np.argmin(t, axis=1)                  # the first of equal distances, like `t < min_t`
            tmin = t[np.arange(cand.size), j]
            qk = tmin / (dx * cmag)
            ok = np.isfinite(qk) & (qk > 0.0) & (qk <= 1.0)
            q[b, cand[ok], k] = qk[ok]
            tri_of[b, cand[ok], k] = near[j[ok]] + 1
    has = (q > 0.0).any(axis=2)
    bi, ci = np.nonzero(has)
    cells = np.stack([bi + 1, (ci & 7) + 1, ((ci >> 3) & 7) + 1, (ci >> 6) + 1], axis=1).astype(np.int32)
    return cells, q[bi, ci].astype(np.float16), tri_of[bi, ci]


def bench_step_cost(steps: int = 200, storage: str = "f16") -> dict:
    """Step time of the 256 x 128 x 128 sphere channel (D = 24, Re 1000) with full-way solid cells and
    with the linear Bouzidi wall, alternating, each on CUDA events over `steps` graph-captured steps
    after 10 warm-up steps."""
    import time

    import torch

    from . import _capi as capi
    from .cases import sphere_channel_case
    from .solver import Geometry, Level

    case = sphere_channel_case(256, 128, 128, diameter=24.0, centre_x=64.0, u_inlet=0.05, re=1000.0)
    t0 = time.time()
    cells, q = sphere_qmap(case.dom, (64.0, 64.0, 64.0), 12.0)
    out = {"workload": "sphere_channel_256x128x128_D24_Re1000", "storage": storage,
           "boundary_cells": int(cells.shape[0]), "links": int((q > 0).sum()), "qmap_s": round(time.time() - t0, 2)}
    g = Geometry(case.dom)
    st = torch.cuda.current_stream()
    for run, bc in (("fullway", capi.OAL_SOLID_FULLWAY), ("bouzidi", capi.OAL_SOLID_BOUZIDI),
                    ("fullway_2", capi.OAL_SOLID_FULLWAY), ("bouzidi_2", capi.OAL_SOLID_BOUZIDI)):
        L = Level(g, storage=storage)
        L.init_equilibrium(case.rho, case.vel)
        if bc == capi.OAL_SOLID_BOUZIDI:
            L.set_bouzidi(cells, q)
        p = capi.default_params(**{f: getattr(case.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
        p.solid_bc = bc
        p.collect_forces = 0
        L.execute_timestep_batch(p, 10, stream=st)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        L.execute_timestep_batch(p, steps, stream=st)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        f = L.state()[0]
        out[run] = {"ms_per_step": round(ms, 4), "mlups": round(256 * 128 * 128 / ms / 1e3, 1),
                    "finite": bool(np.isfinite(f).all())}
        L.close()
    g.close()
    return out


if __name__ == "__main__":
    import json
    import sys

    print(json.dumps(bench_step_cost(int(sys.argv[1]) if len(sys.argv) > 1 else 200)))
