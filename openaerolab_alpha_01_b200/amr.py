"""Block AMR of the D3Q27 cumulant path: levels with 2:1 refinement in space and time.

Host-side mirror of the reference's refined-level machinery (OpenAeroLab, Julia):

* ``refine(parent, blocks)`` — the child level of a set of parent blocks: each refined parent block
  becomes 8 child blocks of the doubled block grid (child block (2p-1) + {0,1} per axis, the
  indexing of amr_coupling.jl:1978-1980 and physics_interpolation.jl:18); blocks sorted like the
  reference's active block tuples (src/geometry/domain.jl:785), 27-entry neighbour table within the
  level (missing neighbours are 0: the pull then interpolates from the parent), periodic wraps per
  axis at the level's resolution.
* ``level_taus(tau_finest, n_levels)`` — the reference's legacy level-viscosity rule
  tau_l - 1/2 = (tau_finest - 1/2) 2^(L-l) (src/solver/physics_scaling.jl:640-700).
* ``Hierarchy`` — ``execute_timestep_batch!`` over a level list (src/solver/solver_control.jl:796-828):
  ``advance(params, n)`` runs n coarse steps of ``recursive_step!`` (one CUDA graph); the levels'
  states are the ``solver.Level`` objects of ``level(l)``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _capi as capi
from ._capi import check, lib
from .solver import BlockDomain, Geometry, Level, _stream_handle


def neighbor_table(coords: np.ndarray, dims: tuple[int, int, int], periodic_mask: int = 0) -> np.ndarray:
    """27-entry neighbour table (27, n), 1-based, 0 = none, direction (dx+1)+3(dy+1)+9(dz+1)
    (domain_topology.jl:919-953), with a wrap on each axis whose bit is set."""
    n = coords.shape[0]
    index = {tuple(c): i + 1 for i, c in enumerate(coords.tolist())}
    nbr = np.zeros((27, n), np.int32)
    for b, (bx, by, bz) in enumerate(coords.tolist()):
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    p = [bx + dx, by + dy, bz + dz]
                    for a in range(3):
                        if periodic_mask & (1 << a):
                            p[a] = (p[a] - 1) % dims[a] + 1
                    nbr[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1), b] = index.get(tuple(p), 0)
    return nbr


def refine(parent: BlockDomain, blocks: Sequence[int]) -> BlockDomain:
    """The child level of the given (0-based) parent blocks."""
    pc = parent.coords
    child = set()
    for b in blocks:
        px, py, pz = (int(v) for v in pc[b])
        for sx in (0, 1):
            for sy in (0, 1):
                for sz in (0, 1):
                    child.add((2 * px - 1 + sx, 2 * py - 1 + sy, 2 * pz - 1 + sz))
    coords = np.array(sorted(child), np.int32).reshape(-1, 3)
    dims = (2 * parent.bx_max, 2 * parent.by_max, 2 * parent.bz_max)
    return BlockDomain(dims[0], dims[1], dims[2], coords, neighbor_table(coords, dims, parent.periodic_mask),
                       periodic_mask=parent.periodic_mask)


def blocks_in_box(dom: BlockDomain, lo: Sequence[float], hi: Sequence[float]) -> list[int]:
    """Blocks of `dom` whose cells intersect the box [lo, hi) (cell units of `dom`, 0-based)."""
    out = []
    for b, (bx, by, bz) in enumerate(dom.coords.tolist()):
        c0 = np.array([(bx - 1) * 8, (by - 1) * 8, (bz - 1) * 8], float)
        if np.all(c0 + 8 > np.asarray(lo, float)) and np.all(c0 < np.asarray(hi, float)):
            out.append(b)
    return out


def level_taus(tau_finest: float, n_levels: int) -> list[float]:
    """Legacy level-viscosity rule: tau_l - 1/2 = (tau_finest - 1/2) 2^(L-l), l = 1..L."""
    return [0.5 + (tau_finest - 0.5) * 2.0 ** (n_levels - 1 - l) for l in range(n_levels)]


def prolong_fields(parent: BlockDomain, child: BlockDomain, rho: np.ndarray, vel: np.ndarray):
    """Child-level (rho, vel) copied from the parent cell that contains each child cell."""
    index = {tuple(c): i for i, c in enumerate(parent.coords.tolist())}
    cell = np.arange(512)
    lx, ly, lz = cell & 7, (cell >> 3) & 7, cell >> 6
    out_r = np.empty((child.n_blocks, 512))
    out_v = np.empty((3, child.n_blocks, 512))
    for b, (bx, by, bz) in enumerate(child.coords.tolist()):
        gx = (bx - 1) * 8 + lx
        gy = (by - 1) * 8 + ly
        gz = (bz - 1) * 8 + lz
        px, py, pz = gx // 2, gy // 2, gz // 2
        pb = np.array([index[(x // 8 + 1, y // 8 + 1, z // 8 + 1)] for x, y, z in zip(px, py, pz)])
        pcell = (px % 8) + 8 * (py % 8) + 64 * (pz % 8)
        out_r[b] = rho[pb, pcell]
        out_v[:, b] = vel[:, pb, pcell]
    return out_r, out_v


class Hierarchy:
    """oal_amr: the levels' geometries and states, stepped by recursive_step!."""

    def __init__(self, domains: Sequence[BlockDomain], storage: str = "f32", device: int = 0):
        self.domains = list(domains)
        self.geoms = [Geometry(d, device) for d in self.domains]
        descs = (capi.AmrLevelDesc * len(domains))()
        for i, (d, g) in enumerate(zip(self.domains, self.geoms)):
            descs[i].geometry = g.handle
            descs[i].dim[0], descs[i].dim[1], descs[i].dim[2] = d.bx_max, d.by_max, d.bz_max
        h = C.c_void_p()
        check(lib().oal_amr_create(len(domains), descs, capi.STORAGE_NAMES[storage], C.byref(h)))
        self.handle = h
        self.levels = []
        for i, (d, g) in enumerate(zip(self.domains, self.geoms)):
            lh = C.c_void_p()
            check(lib().oal_amr_level(h, i, C.byref(lh)))
            self.levels.append(_BorrowedLevel(lh, g, d.n_blocks))

    def level(self, l: int) -> "Level":
        return self.levels[l]

    def advance(self, params: Sequence[capi.StepParams], n_coarse_steps: int, stream=None) -> None:
        arr = (capi.StepParams * len(params))(*params)
        check(lib().oal_amr_advance(self.handle, arr, int(n_coarse_steps), _stream_handle(stream)))

    execute_timestep_batch = advance

    def close(self):
        if getattr(self, "handle", None):
            lib().oal_amr_destroy(self.handle)
            self.handle = None
        for g in getattr(self, "geoms", []):
            g.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _BorrowedLevel(Level):
    """A level owned by the hierarchy (its destroy belongs to oal_amr_destroy)."""

    def __init__(self, handle, geom: Geometry, n_blocks: int):
        self.geom = geom
        self.handle = handle
        self.n_blocks = n_blocks
        self.operator = capi.OAL_OP_CUMULANT_D3Q27
        self.Q = 27

    def close(self):
        self.handle = None
