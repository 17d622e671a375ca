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
