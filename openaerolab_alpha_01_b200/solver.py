"""Host-side mirror of the reference's solver-step and collision-operator interface.

Names follow the reference (OpenAeroLab, Julia):

* ``get_collision_kernel(operator)``  — operator registry (src/collision/physics_kernels.jl:50-75);
  unknown names raise like the reference's ``error()``.
* ``BlockDomain`` + ``build_box`` / ``apply_analytic_sphere_obstacle`` — the block topology of
  ``build_neighbor_table`` (src/geometry/domain_topology.jl:919-953) and the analytic sphere mask
  (src/geometry/domain_generation.jl:132-150).
* ``Level.perform_timestep`` — ``perform_timestep_v2!`` for a level without a parent
  (src/collision/timestep.jl:946-1559): one fused ``stream_collide_cumulant!`` launch, buffers
  swapped by parity (src/solver/solver_control.jl:85-91).
* ``Level.execute_timestep_batch`` — ``execute_timestep_batch!`` (src/solver/solver_control.jl:796-828):
  n steps as one captured CUDA graph.
* ``Level(geom, "entropic")`` — a D3Q39 level stepped by ``stream_collide_entropic_d3q39!``
  (src/collision/kernel_entropic_d3q39.jl:529-3368) with its multiplier warm-start cache
  (``Level.lambda_cache``, src/collision/timestep.jl:1447-1450); parameters from
  ``default_entropic_params`` (timestep.jl:1133-1143).

Arrays use the reference layout flattened to C order: populations ``(Q, n_blocks, 512)``,
density ``(n_blocks, 512)``, velocity ``(3, n_blocks, 512)``; the cell index inside a block is
``x + 8y + 64z``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _capi as capi
from ._capi import check, lib

_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)


def _ptr(a: Optional[np.ndarray], ty):
    if a is None:
        return C.cast(None, ty)
    return a.ctypes.data_as(ty)


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    h = getattr(stream, "cuda_stream", None)
    if h is None:
        raise TypeError("stream must be None, an int handle or a torch.cuda.Stream")
    return int(h)


def get_collision_kernel(operator: str) -> int:
    """Operator id for a reference operator symbol (``"cumulant"``, ``"entropic"``, ``"hrr"``)."""
    out = C.c_int32()
    check(lib().oal_lookup_operator(operator.encode(), C.byref(out)))
    return out.value


def default_step_params(**overrides) -> capi.StepParams:
    """The reference's configuration defaults (src/io/config_loader.jl:1305-1380) with overrides."""
    return capi.default_params(**overrides)


def default_surface_params(**overrides) -> capi.SurfaceParams:
    """The surface-stress mapping's defaults (src/forces/surface.jl:1333-1336, config c_wale)."""
    p = capi.SurfaceParams()
    lib().oal_default_surface_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        if k == "moment_center":
            for i in range(3):
                p.moment_center[i] = float(v[i])
        else:
            setattr(p, k, v)
    return p


def default_entropic_params(**overrides) -> capi.StepParams:
    """Defaults of the D3Q39 entropic operator: ``lambda_param`` is the h-damping sigma
    (ENTROPIC_SIGMA, 0) and ``adaptive_omega4`` the alpha solver (0 bisection, 1 Newton,
    2 approximate, 3 Taylor; config default bisection), as timestep.jl:1133-1143 passes them."""
    p = capi.StepParams()
    lib().oal_default_entropic_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def svv_epsilons(level_id: int, yz_enabled: bool = False, yz_epsilon: float = 0.002, yz_min_level: int = 4,
                 x_enabled: bool = False, x_epsilon: float = 0.002, x_max_level: int = 1) -> dict:
    """The spectral vanishing viscosity strengths of level ``level_id`` (1 = the coarsest), gated as
    timestep.jl:1577-1578 gates them: y-z on levels >= ``yz_min_level``, x on levels <= ``x_max_level``
    (config advanced.numerics.svv_yz / svv_x, config_loader.jl:2317-2332, whose defaults these are).
    Returns the ``svv_x_epsilon`` / ``svv_yz_epsilon`` overrides of the level's step parameters."""
    if yz_min_level < 1:
        raise ValueError("svv_yz.min_level must be >= 1")
    if yz_epsilon < 0 or x_epsilon < 0:
        raise ValueError("SVV epsilons must be >= 0")
    return dict(svv_yz_epsilon=float(yz_epsilon) if yz_enabled and level_id >= yz_min_level else 0.0,
                svv_x_epsilon=float(x_epsilon) if x_enabled and level_id <= x_max_level else 0.0)


@dataclass
class BlockDomain:
    """Block topology and cell fields of one level (host arrays, reference semantics)."""

    bx_max: int
    by_max: int
    bz_max: int
    coords: np.ndarray  # (n, 3) int32, 1-based
    neighbor_table: np.ndarray  # (27, n) int32 C order == Julia (n, 27) column-major, 1-based, 0 = none
    obstacle: Optional[np.ndarray] = None  # (n, 512) uint8
    sponge: Optional[np.ndarray] = None  # (n, 512) float32
    wall_dist: Optional[np.ndarray] = None  # (n, 512) float32
    periodic_mask: int = 0

    @property
    def n_blocks(self) -> int:
        return int(self.coords.shape[0])

    @property
    def shape(self) -> tuple[int, int, int]:
        return (8 * self.bx_max, 8 * self.by_max, 8 * self.bz_max)

    def cell_positions(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """1-based global cell indices (gx, gy, gz), each (n, 512)."""
        cell = np.arange(512)
        lx, ly, lz = cell & 7, (cell >> 3) & 7, cell >> 6
        gx = (self.coords[:, 0:1] - 1) * 8 + lx[None, :] + 1
        gy = (self.coords[:, 1:2] - 1) * 8 + ly[None, :] + 1
        gz = (self.coords[:, 2:3] - 1) * 8 + lz[None, :] + 1
        return gx, gy, gz


def build_box(bx_max: int, by_max: int, bz_max: int, periodic: tuple[bool, bool, bool] = (False, False, False)) -> BlockDomain:
    """All blocks of a box, sorted like the reference, with their 27-entry neighbour table."""
    n = bx_max * by_max * bz_max
    coords = np.zeros((n, 3), dtype=np.int32)
    nbr = np.zeros((27, n), dtype=np.int32)
    mask = (1 if periodic[0] else 0) | (2 if periodic[1] else 0) | (4 if periodic[2] else 0)
    check(lib().oal_build_box_blocks(bx_max, by_max, bz_max, mask, _ptr(coords, _i32p), _ptr(nbr, _i32p)))
    return BlockDomain(bx_max, by_max, bz_max, coords, nbr, periodic_mask=mask)


def apply_analytic_sphere_obstacle(dom: BlockDomain, centre: tuple[float, float, float], radius: float) -> int:
    """Solid mask of a sphere (cell units, cell centres at index - 0.5); returns the solid count."""
    obst = np.zeros((dom.n_blocks, 512), dtype=np.uint8)
    n = C.c_int64()
    check(lib().oal_build_sphere_obstacle(dom.n_blocks, _ptr(dom.coords, _i32p), float(centre[0]), float(centre[1]),
                                          float(centre[2]), float(radius), _ptr(obst, _u8p), C.byref(n)))
    dom.obstacle = obst
    return int(n.value)


def taylor_green_fields(dom: BlockDomain, u0: float, phase: tuple[float, float] = (0.0, 0.0)):
    """2-D Taylor-Green vortex (uniform in z) on a periodic box with the consistent pressure field
    rho = 1 + 3 (u0^2/4)(cos 2kx + cos 2ky), k = 2 pi / nx (tools/tests/q19_octree_step.jl:94)."""
    gx, gy, _ = dom.cell_positions()
    nx = 8 * dom.bx_max
    k = 2.0 * np.pi / nx
    x = gx - 0.5 + phase[0]
    y = gy - 0.5 + phase[1]
    rho = 1.0 + 3.0 * (u0 * u0 / 4.0) * (np.cos(2 * k * x) + np.cos(2 * k * y))
    vel = np.zeros((3,) + rho.shape)
    vel[0] = u0 * np.sin(k * x) * np.cos(k * y)
    vel[1] = -u0 * np.cos(k * x) * np.sin(k * y)
    return np.ascontiguousarray(rho, dtype=np.float64), np.ascontiguousarray(vel, dtype=np.float64)


class Geometry:
    """Device-resident topology of one level (oal_geometry)."""

    def __init__(self, dom: BlockDomain, device: int = 0):
        self.dom = dom
        self._coords = np.ascontiguousarray(dom.coords, dtype=np.int32)
        self._nbr = np.ascontiguousarray(dom.neighbor_table, dtype=np.int32)
        self._obst = None if dom.obstacle is None else np.ascontiguousarray(dom.obstacle, dtype=np.uint8)
        self._sponge = None if dom.sponge is None else np.ascontiguousarray(dom.sponge, dtype=np.float32)
        self._wd = None if dom.wall_dist is None else np.ascontiguousarray(dom.wall_dist, dtype=np.float32)
        nx, ny, nz = dom.shape
        desc = capi.GeometryDesc(dom.n_blocks, nx, ny, nz, _ptr(self._coords, _i32p), _ptr(self._nbr, _i32p),
                                 _ptr(self._obst, _u8p), _ptr(self._sponge, _f32p), _ptr(self._wd, _f32p))
        h = C.c_void_p()
        check(lib().oal_geometry_create(C.byref(desc), device, C.byref(h)))
        self.handle = h

    def blocks(self) -> tuple[int, int, int]:
        """(real, ghost, mask) blocks one member of this geometry occupies in a batch pool."""
        out = (C.c_int64 * 3)()
        check(lib().oal_geometry_blocks(self.handle, out))
        return int(out[0]), int(out[1]), int(out[2])

    def info(self) -> dict:
        out = (C.c_int64 * 5)()
        check(lib().oal_geometry_info(self.handle, out))
        return dict(n_blocks=out[0], fluid_cells=out[1], solid_cells=out[2], boundary_blocks=out[3], mask_blocks=out[4])

    def close(self):
        # the library defers the release while levels built on this geometry are alive
        if getattr(self, "handle", None):
            lib().oal_geometry_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _bouzidi_args(cells, q):
    """(n, block, x, y, z, q binary16) ctypes arguments of a boundary-cell list."""
    cells = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 4)
    qh = np.ascontiguousarray(np.asarray(q, dtype=np.float16).reshape(-1, 27)).view(np.uint16)
    if qh.shape[0] != cells.shape[0]:
        raise ValueError("q must hold 27 values per boundary cell")
    n = int(cells.shape[0])
    cols = [np.ascontiguousarray(cells[:, j]) for j in range(4)]
    _bouzidi_args.keep = (cols, qh)  # alive for the call
    ptrs = [c.ctypes.data_as(_i32p) if n else None for c in cols]
    return (n, *ptrs, qh.ctypes.data_as(C.POINTER(C.c_uint16)) if n else None)


class BouzidiCells:
    """Linear Bouzidi boundary cells for caller-owned arrays (oal_bouzidi_create): `apply(fields)`
    corrects the populations of a step run through oal_stream_collide with OAL_SOLID_BOUZIDI, as
    the reference calls apply_bouzidi_correction! after its kernel."""

    def __init__(self, geom: "Geometry", cells: np.ndarray, q: np.ndarray, storage: str = "f32",
                 q_min_threshold: float = 0.001, ff_fallback: int = 0, limiter_rel_cap: float = 0.0,
                 limiter_abs_cap: float = 0.0):
        self.geom = geom
        h = C.c_void_p()
        args = _bouzidi_args(cells, q)
        check(lib().oal_bouzidi_create(geom.handle, capi.STORAGE_NAMES[storage], *args, float(q_min_threshold),
                                       int(ff_fallback), float(limiter_rel_cap), float(limiter_abs_cap), C.byref(h)))
        self.handle = h

    def apply(self, fields: capi.LevelFields, stream=None) -> None:
        check(lib().oal_bouzidi_apply(self.geom.handle, self.handle, C.byref(fields), _stream_handle(stream)))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().oal_bouzidi_destroy(self.handle)
            self.handle = None


class Level:
    """Library-owned state of one level: ping-pong populations, density, velocity."""

    def __init__(self, geom: Geometry, operator: str = "cumulant", storage: str = "f32", layout: str = "block",
                 rounding: str = "stochastic", math: str = "fast"):
        """layout "block": block-major populations with ghost blocks (default); "dense": the
        padded grid with shared-memory-staged streaming (box levels in FP32/FP16/BF16).
        rounding (FP16/BF16 deviation storage): "stochastic" (default, unbiased in expectation) or
        "nearest". math (D3Q39 entropic levels): "fast" (CUDA's expf / logf, default) or "exact"
        (the software exp / log shared with the CPU oracle: bit-identical to it)."""
        self.geom = geom
        self.storage = capi.STORAGE_NAMES[storage]
        self.operator = get_collision_kernel(operator)
        if rounding not in ("stochastic", "nearest"):
            raise ValueError("rounding must be 'stochastic' or 'nearest'")
        flags = capi.OAL_LEVEL_DENSE if layout == "dense" else 0
        if rounding == "nearest":
            flags |= capi.OAL_LEVEL_ROUND_NEAREST
        if math not in ("fast", "exact"):
            raise ValueError("math must be 'fast' or 'exact'")
        if math == "exact":
            flags |= capi.OAL_LEVEL_EXACT_MATH
        h = C.c_void_p()
        check(lib().oal_level_create_ex(geom.handle, self.operator, self.storage, flags, C.byref(h)))
        self.handle = h
        self.n_blocks = geom.dom.n_blocks
        self.Q = 39 if self.operator == capi.OAL_OP_ENTROPIC_D3Q39 else 27

    # -- state ---------------------------------------------------------------------------
    def init_equilibrium(self, rho: np.ndarray, vel: np.ndarray, compressible_corr: int = 0) -> None:
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        assert rho.size == self.n_blocks * 512 and vel.size == 3 * rho.size
        check(lib().oal_level_init_equilibrium(self.handle, rho.ctypes.data, vel.ctypes.data, compressible_corr))

    def set_state(self, f: np.ndarray, rho: Optional[np.ndarray] = None, vel: Optional[np.ndarray] = None) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        check(lib().oal_level_set_state(self.handle, f.ctypes.data, None if r is None else r.ctypes.data,
                                        None if v is None else v.ctypes.data))

    def state(self):
        nb = self.n_blocks
        f = np.empty((self.Q, nb, 512))
        rho = np.empty((nb, 512))
        vel = np.empty((3, nb, 512))
        check(lib().oal_level_get_state(self.handle, f.ctypes.data, rho.ctypes.data, vel.ctypes.data))
        return f, rho, vel

    def lambda_cache(self, new: Optional[np.ndarray] = None) -> np.ndarray:
        """D3Q39 levels: the 13-multiplier warm-start cache (13, n_blocks, 512), float32, NaN = none;
        `new` replaces it after the read."""
        out = np.empty((13, self.n_blocks, 512), np.float32)
        src = None if new is None else np.ascontiguousarray(new, dtype=np.float32)
        check(lib().oal_level_entropic_lambda(self.handle, out.ctypes.data, None if src is None else src.ctypes.data))
        return out

    # -- stepping ------------------------------------------------------------------------
    def perform_timestep(self, params: capi.StepParams, stream=None) -> None:
        check(lib().oal_level_step(self.handle, C.byref(params), _stream_handle(stream)))

    step = perform_timestep

    def execute_timestep_batch(self, params: capi.StepParams, n_steps: int, stream=None) -> None:
        check(lib().oal_level_advance(self.handle, C.byref(params), int(n_steps), _stream_handle(stream)))

    advance = execute_timestep_batch

    def set_bouzidi(self, cells: np.ndarray, q: np.ndarray, q_min_threshold: float = 0.001, ff_fallback: int = 0,
                    limiter_rel_cap: float = 0.0, limiter_abs_cap: float = 0.0) -> None:
        """Attach the linear Bouzidi boundary cells (solid_bc OAL_SOLID_BOUZIDI): cells (n, 4) int32
        (block, x, y, z) 1-based, q (n, 27) link fractions stored as float16 like the reference's
        q_map. An empty list detaches."""
        args = _bouzidi_args(cells, q)
        check(lib().oal_level_set_bouzidi(self.handle, *args, float(q_min_threshold), int(ff_fallback),
                                          float(limiter_rel_cap), float(limiter_abs_cap)))

    def forces(self) -> np.ndarray:
        out = (C.c_double * 3)()
        check(lib().oal_level_get_forces(self.handle, out))
        return np.array(out[:])

    def set_surface(self, tri: Optional[np.ndarray]) -> None:
        """Attach triangles for the surface-stress mapping: rows (centroid x, y, z, unit outward
        normal x, y, z, area) in cell units; None or an empty array detaches."""
        if tri is None or len(tri) == 0:
            check(lib().oal_level_set_surface(self.handle, 0, None))
            self._surface_n = 0
            return
        t = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 7)
        check(lib().oal_level_set_surface(self.handle, int(t.shape[0]), t.ctypes.data_as(_f32p)))
        self._surface_n = int(t.shape[0])

    def surface_forces(self, params: Optional[capi.SurfaceParams] = None, per_triangle: bool = False):
        """compute_aerodynamics! on the attached triangles: {"pressure", "viscous", "moment"} (FP64),
        and with per_triangle the (n, 6) map (pressure, shear x y z, normal sign, wall distance)."""
        if params is None:
            params = default_surface_params()
        out = (C.c_double * 9)()
        n = getattr(self, "_surface_n", 0)
        per = np.zeros((n, 6), np.float32) if per_triangle else None
        check(lib().oal_level_surface_forces(self.handle, C.byref(params), out,
                                             None if per is None else per.ctypes.data_as(_f32p)))
        v = np.array(out[:])
        res = {"pressure": v[0:3], "viscous": v[3:6], "moment": v[6:9], "total": v[0:3] + v[3:6]}
        if per_triangle:
            res["per_triangle"] = per
        return res

    def forces_async(self, host_buf_ptr: int, stream=None) -> None:
        check(lib().oal_level_get_forces_async(self.handle, host_buf_ptr, _stream_handle(stream)))

    def mass_momentum(self) -> np.ndarray:
        out = (C.c_double * 4)()
        check(lib().oal_level_mass_momentum(self.handle, out))
        return np.array(out[:])

    def set_nscbc(self, enabled: bool = True, all_blocks: bool = False, **kw) -> capi.NscbcParams:
        """The characteristic (NSCBC) outlet after every step (apply_nscbc_outlet!,
        kernel_nscbc_outlet.jl): p_target, sigma_relax, neq_blend as the reference's outlet_nscbc
        settings; all_blocks as the reference's driver launches it (the x = 8 plane of every block)."""
        p = capi.NscbcParams()
        lib().oal_default_nscbc_params(C.byref(p))
        p.enabled = int(bool(enabled))
        p.all_blocks = int(bool(all_blocks))
        for k, v in kw.items():
            if not hasattr(p, k):
                raise AttributeError(k)
            setattr(p, k, v)
        check(lib().oal_level_set_nscbc(self.handle, C.byref(p)))
        return p

    # -- launch tuning (results do not depend on it)
    @property
    def prefetch_ctas(self) -> int:
        v = C.c_int64()
        check(lib().oal_level_get_tuning(self.handle, capi.OAL_TUNE_PREFETCH_CTAS, C.byref(v)))
        return int(v.value)

    @prefetch_ctas.setter
    def prefetch_ctas(self, value: int) -> None:
        check(lib().oal_level_set_tuning(self.handle, capi.OAL_TUNE_PREFETCH_CTAS, int(value)))

    @property
    def persistent(self) -> bool:
        v = C.c_int64()
        check(lib().oal_level_get_tuning(self.handle, capi.OAL_TUNE_PERSISTENT, C.byref(v)))
        return bool(v.value)

    @persistent.setter
    def persistent(self, value: bool) -> None:
        check(lib().oal_level_set_tuning(self.handle, capi.OAL_TUNE_PERSISTENT, int(bool(value))))

    def autotune(self, params: capi.StepParams, n_steps: int = 20) -> dict:
        """Time every candidate launch tuning over n_steps from the current state (restored after
        each) and keep the fastest: {"prefetch_ctas", "persistent": chosen, "candidates":
        [(prefetch, persistent, ms/step)]}."""
        vals = np.zeros(capi.OAL_TUNE_CANDIDATES, np.int64)
        pers = np.zeros(capi.OAL_TUNE_CANDIDATES, np.int32)
        ms = np.zeros(capi.OAL_TUNE_CANDIDATES)
        check(lib().oal_level_autotune(self.handle, C.byref(params), int(n_steps), vals.ctypes.data, pers.ctypes.data,
                                       ms.ctypes.data))
        return {"prefetch_ctas": self.prefetch_ctas, "persistent": self.persistent,
                "candidates": [(int(v), int(q), float(t)) for v, q, t in zip(vals, pers, ms)]}

    def pi_neq(self) -> np.ndarray:
        """Non-equilibrium stress of the current state (compute_pi_neq_kernel!,
        kernel_pi_neq.jl:39-180): float32 (6, n_blocks, 512), xx yy zz xy xz yz, 0 in solid cells."""
        out = np.zeros((6, self.n_blocks, 512), np.float32)
        check(lib().oal_level_pi_neq(self.handle, out.ctypes.data))
        return out

    def layout(self) -> dict:
        out = (C.c_int64 * 6)()
        check(lib().oal_level_layout(self.handle, out))
        return dict(dense=bool(out[0]), PX=out[1], PY=out[2], PZ=out[3], block_stride=out[4], dir_stride=out[5])

    def device_bytes(self) -> int:
        return int(lib().oal_level_device_bytes(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            lib().oal_level_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many cases stepped together: one block pool, one launch per kernel per step for all members,
    n steps per CUDA graph (oal_batch_*). Members join and leave between advances."""

    def __init__(self, storage: str = "f16", max_real_blocks: int = 65536, max_ghost_blocks: int = 16384,
                 max_mask_blocks: int = 4096, max_members: int = 256, device: int = 0):
        self.storage = capi.STORAGE_NAMES[storage]
        h = C.c_void_p()
        check(lib().oal_batch_create(device, self.storage, max_real_blocks, max_ghost_blocks, max_mask_blocks,
                                     max_members, C.byref(h)))
        self.handle = h
        self._geoms = {}

    def add(self, geom: Geometry, params: capi.StepParams, rho: np.ndarray, vel: np.ndarray) -> int:
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        m = C.c_int32()
        check(lib().oal_batch_add(self.handle, geom.handle, C.byref(params), rho.ctypes.data, vel.ctypes.data,
                                  C.byref(m)))
        self._geoms[m.value] = geom
        return m.value

    def try_add(self, geom: Geometry, params: capi.StepParams, rho: np.ndarray, vel: np.ndarray) -> Optional[int]:
        """add(), or None when the pool has no room (OAL_E_ADMISSION)."""
        try:
            return self.add(geom, params, rho, vel)
        except capi.OALError as e:
            if e.status == capi.OAL_E_ADMISSION:
                return None
            raise

    def remove(self, member: int) -> None:
        check(lib().oal_batch_remove(self.handle, member))
        self._geoms.pop(member, None)

    def set_params(self, member: int, params: capi.StepParams) -> None:
        check(lib().oal_batch_set_params(self.handle, member, C.byref(params)))

    def advance(self, n_steps: int, stream=None) -> None:
        check(lib().oal_batch_advance(self.handle, int(n_steps), _stream_handle(stream)))

    def set_bouzidi(self, member: int, cells: np.ndarray, q: np.ndarray, q_min_threshold: float = 0.001,
                    ff_fallback: int = 0, limiter_rel_cap: float = 0.0, limiter_abs_cap: float = 0.0) -> None:
        """A member's linear Bouzidi boundary cells, as Level.set_bouzidi (block indices of the
        member's geometry)."""
        args = _bouzidi_args(cells, q)
        check(lib().oal_batch_set_bouzidi(self.handle, int(member), *args, float(q_min_threshold), int(ff_fallback),
                                          float(limiter_rel_cap), float(limiter_abs_cap)))

    @property
    def prefetch_ctas(self) -> int:
        v = C.c_int64()
        check(lib().oal_batch_get_tuning(self.handle, capi.OAL_TUNE_PREFETCH_CTAS, C.byref(v)))
        return int(v.value)

    @prefetch_ctas.setter
    def prefetch_ctas(self, value: int) -> None:
        check(lib().oal_batch_set_tuning(self.handle, capi.OAL_TUNE_PREFETCH_CTAS, int(value)))

    @property
    def persistent(self) -> bool:
        v = C.c_int64()
        check(lib().oal_batch_get_tuning(self.handle, capi.OAL_TUNE_PERSISTENT, C.byref(v)))
        return bool(v.value)

    @persistent.setter
    def persistent(self, value: bool) -> None:
        check(lib().oal_batch_set_tuning(self.handle, capi.OAL_TUNE_PERSISTENT, int(bool(value))))

    def autotune(self, n_steps: int = 20) -> dict:
        """The pool's autotuner (oal_batch_autotune): the members' state is restored afterwards."""
        vals = np.zeros(capi.OAL_TUNE_CANDIDATES, np.int64)
        pers = np.zeros(capi.OAL_TUNE_CANDIDATES, np.int32)
        ms = np.zeros(capi.OAL_TUNE_CANDIDATES)
        check(lib().oal_batch_autotune(self.handle, int(n_steps), vals.ctypes.data, pers.ctypes.data, ms.ctypes.data))
        return {"prefetch_ctas": self.prefetch_ctas, "persistent": self.persistent,
                "candidates": [(int(v), int(q), float(t)) for v, q, t in zip(vals, pers, ms)]}

    def state(self, member: int):
        nb = self._geoms[member].dom.n_blocks
        f = np.empty((27, nb, 512)); rho = np.empty((nb, 512)); vel = np.empty((3, nb, 512))
        check(lib().oal_batch_get_state(self.handle, member, f.ctypes.data, rho.ctypes.data, vel.ctypes.data))
        return f, rho, vel

    def forces(self, member: int) -> np.ndarray:
        out = (C.c_double * 3)()
        check(lib().oal_batch_get_forces(self.handle, member, out))
        return np.array(out[:])

    def mass_momentum(self, member: int) -> np.ndarray:
        out = (C.c_double * 4)()
        check(lib().oal_batch_mass_momentum(self.handle, member, out))
        return np.array(out[:])

    def info(self) -> dict:
        out = (C.c_int64 * 8)()
        check(lib().oal_batch_info(self.handle, out))
        keys = ["members", "real_used", "ghost_used", "mask_used", "real_cap", "ghost_cap", "mask_cap", "bytes"]
        return dict(zip(keys, [int(v) for v in out]))

    def close(self):
        if getattr(self, "handle", None):
            lib().oal_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kinetic_energy(rho: np.ndarray, vel: np.ndarray, obstacle: Optional[np.ndarray] = None) -> float:
    """Sum of rho |u|^2 / 2 over fluid cells (tools/tests/q19_octree_step.jl:17-24)."""
    ke = 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
    if obstacle is not None:
        ke = np.where(obstacle != 0, 0.0, ke)
    return float(ke.sum())
