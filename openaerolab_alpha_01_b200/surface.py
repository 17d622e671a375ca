"""Surface-stress force mapping on a D3Q27 level (the reference's compute_aerodynamics!,
src/forces/surface.jl:1577-1587, default Prandtl force method).

* ``sphere_mesh`` — a closed latitude-longitude triangulation of a sphere (outward normals),
  rows of the C ABI's triangle table (centroid, unit normal, area) in cell units.
* ``triangle_table`` — the same table from triangle vertices (n, 3, 3).
* ``compute_aerodynamics`` — map the stresses on a level's current macros and integrate them:
  pressure and viscous forces, moment, and the coefficients for a reference area and speed.
"""
from __future__ import annotations

import numpy as np

from .solver import Level, default_surface_params


def triangle_table(verts: np.ndarray) -> np.ndarray:
    """(n, 7) rows: centroid, unit normal (right-hand order of the vertices), area."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 3, 3)
    c = v.mean(axis=1)
    cr = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    a2 = np.linalg.norm(cr, axis=1)
    keep = a2 > 0
    n = cr[keep] / a2[keep, None]
    return np.ascontiguousarray(np.concatenate([c[keep], n, 0.5 * a2[keep, None]], axis=1), dtype=np.float32)


def sphere_mesh(centre, radius: float, n_theta: int = 48, n_phi: int = 96) -> np.ndarray:
    """Closed triangulated sphere with outward normals (the pole caps as triangle fans)."""
    th = np.linspace(0.0, np.pi, n_theta + 1)
    ph = np.linspace(0.0, 2.0 * np.pi, n_phi + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    X = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1) * radius + np.asarray(centre, float)
    tris = []
    for i in range(n_theta):
        for j in range(n_phi):
            a, b, c, d = X[i, j], X[i + 1, j], X[i + 1, j + 1], X[i, j + 1]
            if i > 0:
                tris.append((a, b, d))  # outward: (b - a) x (d - a) points away from the centre
            if i < n_theta - 1:
                tris.append((b, c, d))
    t = triangle_table(np.array(tris))
    # orient every normal outward
    out = np.sum((t[:, 0:3] - np.asarray(centre, float)) * t[:, 3:6], axis=1) < 0
    t[out, 3:6] *= -1
    return t


def compute_aerodynamics(level: Level, tri: np.ndarray | None = None, tau: float | None = None,
                         u_ref: float = 0.05, area_ref: float = 1.0, rho_ref: float = 1.0, per_triangle: bool = False,
                         **params) -> dict:
    """Surface forces on the level's current state; `tri` attaches a new triangle table first.
    Coefficients C = F / (1/2 rho_ref u_ref^2 area_ref) (lattice units)."""
    if tri is not None:
        level.set_surface(tri)
    if tau is not None:
        params["tau"] = tau
    r = level.surface_forces(default_surface_params(**params), per_triangle=per_triangle)
    q = 0.5 * rho_ref * u_ref * u_ref * area_ref
    r["coefficients"] = r["total"] / q
    r["pressure_coefficients"] = r["pressure"] / q
    r["viscous_coefficients"] = r["viscous"] / q
    return r
