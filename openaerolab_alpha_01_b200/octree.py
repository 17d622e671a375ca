"""D3Q19 octree solver on the GPU: a single periodic level behind the reference's OctreeQ19 API.

Mirrors (OpenAeroLab src/octree_q19, Julia):
    MeshSpec(domain, periodic=(true,)*3, levels=1) + generate(Tri[], spec)   -> PeriodicBox
        generator.jl:270-350 (octs of level 1 in Morton order, onbr with periodic wrap)
    test_case_config(spec; nu_lattice, u_lattice, velocity, hrr_sigma, sgs, precision, body_force)
        config.jl:306-335, lattice scaling config.jl:328-335           -> test_case_config / CaseConfig
    State(mesh, cfg, T)                                                  -> State
    initialise!(st, init; nonequilibrium) / initialise_uniform!          -> State.initialise / initialise_uniform
        state.jl:267-330
    advance!(st)                                                         -> State.advance
        run.jl:6-11, stream.jl:280-380
    total_mass / total_momentum                                          -> State.total_mass / total_momentum
        state.jl:333-356

The step runs in liboal (include/oal.h, oal_q19_*); `init` is evaluated on the host as in the
reference. `init(x, y, z)` takes arrays of slot centres (metres) and returns (rho, ux, uy, uz)
arrays (numpy broadcasting: the reference's per-point function written with numpy functions).
A level with domain faces and a body comes from `generate(tri, MeshSpec(...))` (one level, the
reference's generator restated natively); refined meshes are refused (OAL_E_UNSUPPORTED).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from ._capi import check, lib

SGS_CODES = {"none": capi.OAL_Q19_SGS_NONE, "wale": capi.OAL_Q19_SGS_WALE,
             "smagorinsky": capi.OAL_Q19_SGS_SMAGORINSKY, "vreman": capi.OAL_Q19_SGS_VREMAN}
_PRECISION = {np.dtype(np.float32): capi.OAL_STORE_F32, np.dtype(np.float64): capi.OAL_STORE_F64}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class PeriodicBox:
    """Level 1 of a periodic box of n0 x n1 x n2 cells (even counts) with cell size dx."""

    def __init__(self, n0: int, n1: int | None = None, n2: int | None = None, dx: float = 1.0):
        n1 = n0 if n1 is None else n1
        n2 = n0 if n2 is None else n2
        self.n = (int(n0), int(n1), int(n2))
        self.dx = float(dx)
        self.nocts = (n0 // 2) * (n1 // 2) * (n2 // 2)
        self.origin = np.zeros((self.nocts, 3), np.int32)   # reference (3, nocts)
        self.onbr = np.zeros((self.nocts, 27), np.int32)    # reference (27, nocts), 1-based
        check(lib().oal_q19_periodic_box(n0, n1, n2, _ptr(self.origin), _ptr(self.onbr)))
        self.counts = {"fluid_total": n0 * n1 * n2, "octs": self.nocts}

    def slot_cells(self) -> np.ndarray:
        """(nocts, 3, 8) integer cell of every slot (octree.jl slot_offset: k-1 = x + 2y + 4z)."""
        k = np.arange(8)
        off = np.stack([k & 1, (k >> 1) & 1, (k >> 2) & 1])  # (3, 8)
        return self.origin[:, :, None] + off[None]

    def slot_centres(self) -> np.ndarray:
        """(nocts, 3, 8) slot centres in metres (octree.jl:113-116)."""
        return (self.slot_cells() + 0.5) * self.dx


@dataclass
class Region:
    """A refinement region (generator.jl:10-16): kind "box" (lo..hi), "sphere" (centre, radius) or
    "cylinder" (axis lo -> hi, radius), refined up to `level`."""
    kind: str
    level: int
    lo: tuple = (0.0, 0.0, 0.0)
    hi: tuple = (0.0, 0.0, 0.0)
    centre: tuple = (0.0, 0.0, 0.0)
    radius: float = 0.0


@dataclass
class SurfaceLevel:
    """A box with its own surface level (generator.jl:18-21): cells whose centre lies in [lo, hi]
    are refined to max(MeshSpec.surface_level, level) in the surface band."""
    level: int
    lo: tuple
    hi: tuple


@dataclass
class MeshSpec:
    """MeshSpec of the reference (generator.jl:21-36): the domain in metres, the periodic axes, the
    number of levels and the finest cell size, the surface bands, regions and the condition of each
    domain face (-x +x -y +y -z +z), per-box surface levels and cavity sealing."""
    domain: tuple
    periodic: tuple = (False, False, False)
    levels: int = 1
    dx_finest: float = 1.0
    surface_level: int = 0
    band_fine: int = 8
    band: int = 6
    wake_length: float = 0.0
    wake_level_offset: int = 1
    wake_margin: float = 0.1
    regions: tuple = ()
    faces: tuple = ("inlet", "outlet", "slip", "slip", "slip", "slip")
    seal_cavities: bool = False
    surface_levels: tuple = ()   # SurfaceLevel(level, lo, hi): boxes with their own surface level

    def native(self):
        s = capi.Q19MeshSpec()
        check(lib().oal_q19_default_mesh_spec(C.byref(s)))
        for a in range(3):
            s.domain[a] = float(self.domain[a])
            s.periodic[a] = int(bool(self.periodic[a]))
        s.dx = float(self.dx_finest)
        s.levels = int(self.levels)
        s.surface_level = int(self.surface_level)
        s.band_fine = int(self.band_fine)
        s.band = int(self.band)
        s.wake_length = float(self.wake_length)
        s.wake_level_offset = int(self.wake_level_offset)
        s.wake_margin = float(self.wake_margin)
        s.seal_cavities = int(bool(self.seal_cavities))
        for f in range(6):
            s.faces[f] = capi.Q19_FACE_NAMES[self.faces[f]]
        regs = (capi.Q19Region * max(len(self.regions), 1))()
        for i, r in enumerate(self.regions):
            regs[i].kind = {"box": 0, "sphere": 1, "cylinder": 2}[r.kind]
            regs[i].level = int(r.level)
            for a in range(3):
                regs[i].lo[a], regs[i].hi[a], regs[i].centre[a] = r.lo[a], r.hi[a], r.centre[a]
            regs[i].radius = float(r.radius)
        s.nregions = len(self.regions)
        s.regions = C.cast(regs, C.c_void_p) if self.regions else None
        sl = (capi.Q19SurfaceLevel * max(len(self.surface_levels), 1))()
        for i, b in enumerate(self.surface_levels):
            sl[i].level = int(b.level)
            for a in range(3):
                sl[i].lo[a], sl[i].hi[a] = float(b.lo[a]), float(b.hi[a])
        s.nsurface_levels = len(self.surface_levels)
        s.surface_levels = C.cast(sl, C.c_void_p) if self.surface_levels else None
        return s, (regs, sl)


_DESC_ARRAYS = [("origin", np.int32, (3,)), ("real", np.uint8, ()), ("onbr", np.int32, (27,)),
                ("kind", np.uint8, (8,)), ("face", np.uint8, (8,)), ("special", np.uint32, (8,)),
                ("cutidx", np.int32, (8,))]
_CUT_ARRAYS = [("cut_dir", np.uint8), ("cut_q", np.float32), ("cut_tri", np.int32), ("cut_partner", np.uint8)]
_TRANSFER_ARRAYS = [("ghost_slot", "nghost", np.int32, ()), ("ghost_donor", "nghost", np.int32, (64,)),
                    ("ghost_w", "nghost", np.float32, (64,)), ("restrict_slot", "nrestrict", np.int32, ()),
                    ("restrict_src", "nrestrict", np.int32, (64,)), ("restrict_cubic", "nrestrict", np.uint8, ())]
COUNT_NAMES = ("octs", "n0", "n1", "n2", "fluid_total", "solid", "boundary", "wall_cells", "cut_links",
               "leak_cells", "missing_partner_links", "unreached_triangles", "special_slots", "real_octs",
               "ghosts_listed", "restricted")


class Mesh:
    """One octree level with domain faces and a body: the reference's OctLevel arrays as numpy arrays
    in its memory order (C-order shapes: kind (nocts, 8) is Julia's (8, nocts))."""

    def __init__(self, arrays: dict, n, dx, faces, ntri, counts=None):
        self.__dict__.update(arrays)
        self.nocts = int(self.onbr.shape[0])
        self.n = tuple(int(v) for v in n)
        self.dx = float(dx)
        self.faces = tuple(int(f) for f in faces)
        self.ntri = int(ntri)
        self.counts = counts or {}

    slot_cells = PeriodicBox.slot_cells
    slot_centres = PeriodicBox.slot_centres

    def oct_index(self) -> dict:
        """origin -> 0-based oct (built once)."""
        if getattr(self, "_octidx", None) is None:
            self._octidx = {tuple(int(v) for v in o): i for i, o in enumerate(self.origin)}
        return self._octidx

    @classmethod
    def from_native(cls, handle, level: int = 1) -> "Mesh":
        d = capi.Q19LevelDesc()
        check(lib().oal_q19_mesh_level_desc(handle, level, C.byref(d)))
        cnt = (C.c_int64 * 16)()
        check(lib().oal_q19_mesh_counts(handle, level, cnt))
        no = d.nocts
        arrays = {}
        for name, dt, shape in _DESC_ARRAYS:
            n = no * int(np.prod(shape))
            ptr = getattr(d, name)
            if not n or not ptr:  # a level without octs
                arrays[name] = np.zeros((no,) + shape, dt)
                continue
            buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(ptr)
            arrays[name] = np.frombuffer(buf, dt).reshape((no,) + shape).copy()
        def view(ptr, n, dt):
            if not n or not ptr:
                return np.zeros(n if ptr else 0, dt)
            return np.frombuffer((C.c_char * (n * np.dtype(dt).itemsize)).from_address(ptr), dt).copy()

        for name, dt in _CUT_ARRAYS:
            arrays[name] = view(getattr(d, name), d.nlinks, dt)
        for name, cname, dt, shape in _TRANSFER_ARRAYS:
            cnt_ = getattr(d, cname)
            arrays[name] = view(getattr(d, name), cnt_ * int(np.prod(shape)), dt).reshape((cnt_,) + shape)
        arrays["cut_slot"] = view(d.cut_slot, d.ncut, np.int32)
        arrays["cut_off"] = view(d.cut_off, d.ncut + 1, np.int32)
        if arrays["cut_off"].size == 0:
            arrays["cut_off"] = np.ones(1, np.int32)
        counts = {k: int(v) for k, v in zip(COUNT_NAMES, cnt[:len(COUNT_NAMES)])}
        return cls(arrays, (counts["n0"], counts["n1"], counts["n2"]), 0.0, list(d.faces), d.ntri, counts)

    def desc(self) -> capi.Q19LevelDesc:
        """A level descriptor pointing at this mesh's arrays (valid while the mesh lives)."""
        d = capi.Q19LevelDesc()
        d.nocts = self.nocts
        for name, _, _ in _DESC_ARRAYS:
            setattr(d, name, getattr(self, name).ctypes.data)
        d.ncut = int(self.cut_slot.shape[0])
        d.nlinks = int(self.cut_dir.shape[0])
        for name in ("cut_slot", "cut_off", "cut_dir", "cut_q", "cut_tri", "cut_partner"):
            a = getattr(self, name)
            setattr(d, name, a.ctypes.data if a.size else None)
        d.ntri = self.ntri
        for f in range(6):
            d.faces[f] = self.faces[f]
        for name, cname, _, _ in _TRANSFER_ARRAYS:
            a = getattr(self, name, None)
            n = 0 if a is None else int(a.shape[0])
            setattr(d, cname, n)
            setattr(d, name, a.ctypes.data if n else None)
        return d


class OctMesh:
    """The levels of an octree mesh (the reference's OctMesh): `levels[l - 1]` is level l."""

    def __init__(self, levels, counts, spec):
        self.levels = levels
        self.counts = counts
        self.spec = spec

    @property
    def nlevels(self) -> int:
        return len(self.levels)

    def locate_leaf(self, p):
        """(level, 0-based slot) of the real leaf (fluid, or solid) containing point p, or (0, -1)
        (octree.jl:248-262)."""
        for l in range(self.nlevels, 0, -1):
            lv = self.levels[l - 1]
            c = [int(np.floor(p[a] / lv.dx)) for a in range(3)]
            if any(c[a] < 0 or c[a] >= lv.n[a] for a in range(3)):
                return 0, -1
            key = (c[0] & ~1, c[1] & ~1, c[2] & ~1)
            o = lv.oct_index().get(key)
            if o is None or not lv.real[o]:
                continue
            s = 8 * o + (c[0] & 1) + 2 * (c[1] & 1) + 4 * (c[2] & 1)
            if lv.kind[o, s % 8] == capi.OAL_Q19_K_COVERED:
                continue
            return l, s
        return 0, -1

    def work_W(self) -> int:
        """Fluid cell updates per coarse step, sum over levels of fluid_l 2^(l-1) (run.jl:99)."""
        return sum(m.counts["fluid_total"] << l for l, m in enumerate(self.levels))


def generate(tri, spec: MeshSpec) -> OctMesh:
    """The reference's generate(tri, spec): triangles (ntri, 3, 3) in metres."""
    t = np.ascontiguousarray(np.asarray(tri, np.float64).reshape(-1, 3, 3))
    h = C.c_void_p()
    native, _keep = spec.native()
    check(lib().oal_q19_mesh_generate(t.ctypes.data_as(C.c_void_p) if t.size else None, t.shape[0],
                                      C.byref(native), C.byref(h)))
    try:
        L = lib().oal_q19_mesh_levels(h)
        levels = [Mesh.from_native(h, l) for l in range(1, L + 1)]
        cnt = (C.c_int64 * 16)()
        check(lib().oal_q19_mesh_counts(h, 0, cnt))
        seal = (C.c_int64 * 2)()
        check(lib().oal_q19_mesh_seal_counts(h, seal))
    finally:
        lib().oal_q19_mesh_destroy(h)
    for l, m in enumerate(levels, start=1):
        m.level = l
        m.dx = float(spec.dx_finest) * 2.0 ** (L - l)
        m.domain = tuple(v * m.dx for v in m.n)
    counts = {k: int(v) for k, v in zip(COUNT_NAMES, cnt[:len(COUNT_NAMES)])}
    counts["sealed_cells"], counts["cavity_unbracketed_parity_cells"] = int(seal[0]), int(seal[1])
    counts["per_level"] = [m.counts for m in levels]
    return OctMesh(levels, counts, spec)


def box_triangles(lo, hi) -> np.ndarray:
    """A closed box of 12 outward-facing triangles (the reference tests' box_tris)."""
    v = np.array([(x, y, z) for z in (lo[2], hi[2]) for y in (lo[1], hi[1]) for x in (lo[0], hi[0])], np.float64)
    faces = ((0, 2, 6, 4), (1, 5, 7, 3), (0, 4, 5, 1), (2, 3, 7, 6), (0, 1, 3, 2), (4, 6, 7, 5))
    tri = []
    for f in faces:
        tri.append((v[f[0]], v[f[1]], v[f[2]]))
        tri.append((v[f[0]], v[f[2]], v[f[3]]))
    return np.array(tri)


@dataclass
class CaseConfig:
    nu_lattice: float = 0.01
    u_lattice: float = 0.08
    velocity: float = 1.0
    hrr_sigma: float = 1.0
    sgs: str = "none"
    c_wale: float = 0.5
    c_smagorinsky: float = 0.1
    body_force: tuple = (0.0, 0.0, 0.0)
    precision: type = np.float32
    dx: float = 1.0
    extra: dict = field(default_factory=dict)

    def level_nu(self, level: int = 1, levels: int = 1) -> float:
        """Lattice viscosity of level `level` of `levels` (config.jl:309, 328-335): the physical
        viscosity times dt_l / dx_l^2, both scaling with 2^(L - l) from the finest level."""
        nu_phys = self.nu_lattice * self.velocity * self.dx / self.u_lattice
        vs = self.velocity / self.u_lattice
        dtf = self.dx / vs
        s = 2.0 ** (levels - level)
        return nu_phys * (dtf * s) / (self.dx * s) ** 2

    def params(self, level: int = 1, levels: int = 1) -> capi.Q19Params:
        """The step parameters of level `level`: its viscosity, the body force in its lattice units
        (x 2^(L - l), stream.jl:291-293) and the momentum-exchange scale 8^(1 - l) (coupling.jl:246)."""
        if self.sgs not in SGS_CODES:
            raise ValueError(f"unknown sgs model {self.sgs!r}")
        p = capi.Q19Params()
        check(lib().oal_q19_default_params(C.byref(p)))
        p.nu = self.level_nu(level, levels)
        p.u_inlet[0] = self.u_lattice          # st.u_inlet * inlet_dir, inlet along +x (state.jl:255)
        p.force_scale = 8.0 ** (1 - level)
        p.sgs = SGS_CODES[self.sgs]
        p.c_wale = self.c_wale
        p.c_smagorinsky = self.c_smagorinsky
        p.hrr_sigma = self.hrr_sigma
        fs = 2.0 ** (levels - level)
        for a in range(3):
            p.body_force[a] = float(self.body_force[a] * fs)
        return p


def test_case_config(box, nu_lattice: float = 0.01, u_lattice: float = 0.08, velocity: float = 1.0,
                     hrr_sigma: float = 1.0, sgs: str = "none", precision=np.float32,
                     body_force=(0.0, 0.0, 0.0)) -> CaseConfig:
    return CaseConfig(nu_lattice=nu_lattice, u_lattice=u_lattice, velocity=velocity, hrr_sigma=hrr_sigma, sgs=sgs,
                      body_force=tuple(body_force), precision=precision, dx=box.dx)


test_case_config.__test__ = False  # a configuration factory, not a pytest test


class State:
    """The level's populations, velocity and density on the GPU (two buffers, swapped per step)."""

    def __init__(self, mesh, cfg: CaseConfig, precision=None, device: int = 0):
        """`mesh`: a PeriodicBox, one level (Mesh) or an OctMesh; an OctMesh of several levels is
        stepped as the reference's step_recursive! (the coarse step of advance!)."""
        self.config_sha = str(getattr(mesh, "config_sha", "") or "")
        self.stl_sha = str(getattr(mesh, "stl_sha", "") or "")
        if isinstance(mesh, OctMesh) and mesh.nlevels == 1:
            mesh = mesh.levels[0]
        self.mesh = mesh
        self.cfg = cfg
        self.dtype = np.dtype(precision or cfg.precision)
        if self.dtype not in _PRECISION:
            raise ValueError("precision must be float32 or float64")
        self.step = 0
        self.mass0 = float("nan")
        self.forces = np.zeros(3)
        self._tree = None
        h = C.c_void_p()
        if isinstance(mesh, OctMesh):
            L = mesh.nlevels
            self.level_meshes = mesh.levels
            self.level_params = [cfg.params(l, L) for l in range(1, L + 1)]
            self._descs = (capi.Q19LevelDesc * L)(*[m.desc() for m in mesh.levels])
            check(lib().oal_q19_octree_create(device, _PRECISION[self.dtype], L, self._descs, C.byref(h)))
            self._tree = h
            self._h = None
        else:
            self.level_meshes = [mesh]
            self.level_params = [cfg.params()]
            if isinstance(mesh, Mesh):
                self._desc = mesh.desc()
                check(lib().oal_q19_level_create_desc(device, _PRECISION[self.dtype], C.byref(self._desc), C.byref(h)))
            else:
                check(lib().oal_q19_level_create(device, _PRECISION[self.dtype], mesh.nocts, _ptr(mesh.onbr), C.byref(h)))
            self._h = h

    @property
    def params(self):
        """The parameters of the single level (the finest level's of a refined mesh)."""
        return self.level_params[-1]

    @params.setter
    def params(self, p):
        self.level_params[-1] = p

    @property
    def nlevels(self) -> int:
        return len(self.level_meshes)

    def _level_handle(self, level: int):
        if self._tree is None:
            return self._h
        h = C.c_void_p()
        check(lib().oal_q19_octree_level(self._tree, level, C.byref(h)))
        return h

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().oal_q19_level_destroy(self._h)
            self._h = None
        if getattr(self, "_tree", None) is not None and self._tree.value:
            lib().oal_q19_octree_destroy(self._tree)
            self._tree = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- initial state
    def _upload(self, rho, u, du):
        if self._tree is not None:
            return self._upload_levels([(rho, u, du)] if not isinstance(rho, list) else list(zip(rho, u, du)))
        rho = np.ascontiguousarray(rho, self.dtype)
        u = np.ascontiguousarray(u, self.dtype)
        du = None if du is None else np.ascontiguousarray(du, self.dtype)
        check(lib().oal_q19_level_initialise(self._h, C.byref(self.params), _ptr(rho), _ptr(u), _ptr(du)))
        self.step = 0
        self.mass0 = self.total_mass()

    def _upload_levels(self, fields):
        keep = [tuple(None if a is None else np.ascontiguousarray(a, self.dtype) for a in f) for f in fields]
        L = self.nlevels
        P = (capi.Q19Params * L)(*self.level_params)
        ptrs = [(C.c_void_p * L)(*[(k[i].ctypes.data if k[i] is not None else None) for k in keep]) for i in range(3)]
        check(lib().oal_q19_octree_initialise(self._tree, P, ptrs[0], ptrs[1],
                                              ptrs[2] if any(k[2] is not None for k in keep) else None))
        self.step = 0
        self.mass0 = self.total_mass()

    def initial_fields(self, init, nonequilibrium: bool = True, level: int = None):
        """(rho (nocts,8), u (nocts,3,8), du (nocts,9,8) or None) of `init` at the slot centres, in the
        level's precision, as state.jl:267-305 forms them (du over one cell, evaluated in Float64).
        A refined mesh gives one such tuple per level (level=None) or that of `level`."""
        if self._tree is not None and level is None:
            return [self.initial_fields(init, nonequilibrium, l) for l in range(1, self.nlevels + 1)]
        mesh = self.level_meshes[(level or 1) - 1]
        p = mesh.slot_centres()
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        rho, ux, uy, uz = (np.broadcast_to(np.asarray(v, np.float64), x.shape) for v in init(x, y, z))
        u = np.stack([ux, uy, uz], 1)
        du = None
        if nonequilibrium:
            h = mesh.dx / 2
            du = np.zeros((mesh.nocts, 9, 8), np.float64)
            for a in range(3):
                e = [0.0, 0.0, 0.0]
                e[a] = h
                up = init(x + e[0], y + e[1], z + e[2])
                um = init(x - e[0], y - e[1], z - e[2])
                for b in range(3):
                    du[:, 3 * a + b] = np.asarray(up[b + 1], np.float64) - np.asarray(um[b + 1], np.float64)
            du = du.astype(self.dtype)
        return rho.astype(self.dtype), u.astype(self.dtype), du

    def initialise(self, init, nonequilibrium: bool = True):
        f = self.initial_fields(init, nonequilibrium)
        if self._tree is not None:
            self._upload_levels(f)
        else:
            self._upload(*f)
        return self

    def initialise_uniform(self, rho0: float, ux0: float, uy0: float, uz0: float):
        fields = []
        for m in self.level_meshes:
            rho = np.full((m.nocts, 8), rho0, self.dtype)
            u = np.empty((m.nocts, 3, 8), self.dtype)
            u[:, 0], u[:, 1], u[:, 2] = self.dtype.type(ux0), self.dtype.type(uy0), self.dtype.type(uz0)
            fields.append((rho, u, None))
        if self._tree is not None:
            self._upload_levels(fields)
        else:
            self._upload(*fields[0])
        return self

    # -- stepping
    def advance(self, n: int = 1, stream=None, collect: bool = False):
        """n coarse steps (advance! n times); with `collect` the last coarse step's momentum exchange
        (every level and sub-step) is kept in `forces` (coarse-lattice units, FP64)."""
        st = None if stream is None else C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else stream)
        if self._tree is not None:
            P = (capi.Q19Params * self.nlevels)(*self.level_params)
            check(lib().oal_q19_octree_advance(self._tree, P, int(n), int(bool(collect)), st))
        else:
            check(lib().oal_q19_level_advance(self._h, C.byref(self.params), int(n), int(bool(collect)), st))
        self.step += n
        if collect and n > 0:
            out = (C.c_double * 3)()
            if self._tree is not None:
                check(lib().oal_q19_octree_forces(self._tree, out, None))
            else:
                check(lib().oal_q19_level_forces(self._h, out, None))
            self.forces = np.array(out[:])
        return self

    def forces_per_triangle(self) -> np.ndarray:
        ntri = max(max(getattr(m, "ntri", 0) for m in self.level_meshes), 1)
        out = np.zeros((ntri, 3))
        if self._tree is not None:
            check(lib().oal_q19_octree_forces(self._tree, None, out.ctypes.data_as(C.c_void_p)))
        else:
            check(lib().oal_q19_level_forces(self._h, None, out.ctypes.data_as(C.c_void_p)))
        return out

    # -- read-out
    def state(self, level: int = 1):
        """(f, u, rho) of `level` in the reference's layout (host copies)."""
        no = self.level_meshes[level - 1].nocts
        f = np.empty((no, 19, 8), self.dtype)
        u = np.empty((no, 3, 8), self.dtype)
        rho = np.empty((no, 8), self.dtype)
        check(lib().oal_q19_level_get_state(self._level_handle(level), _ptr(f), _ptr(u), _ptr(rho)))
        return f, u, rho

    def buffer(self, which: int, level: int = 1):
        """(f, u, rho) of buffer `which` of `level`: 0 the current state, 1 the other one (the
        previous step's; the reference's S.g, S.v, S.rhob)."""
        no = self.level_meshes[level - 1].nocts
        f = np.empty((no, 19, 8), self.dtype)
        u = np.empty((no, 3, 8), self.dtype)
        rho = np.empty((no, 8), self.dtype)
        check(lib().oal_q19_level_get_buffer(self._level_handle(level), int(which), _ptr(f), _ptr(u), _ptr(rho)))
        return f, u, rho

    def set_buffer(self, which: int, f, u, rho, level: int = 1):
        f = np.ascontiguousarray(f, self.dtype)
        u = np.ascontiguousarray(u, self.dtype)
        rho = np.ascontiguousarray(rho, self.dtype)
        check(lib().oal_q19_level_set_buffer(self._level_handle(level), int(which), _ptr(f), _ptr(u), _ptr(rho)))

    def set_state(self, f, u, rho, level: int = 1):
        f = np.ascontiguousarray(f, self.dtype)
        u = np.ascontiguousarray(u, self.dtype)
        rho = np.ascontiguousarray(rho, self.dtype)
        check(lib().oal_q19_level_set_state(self._level_handle(level), _ptr(f), _ptr(u), _ptr(rho)))

    def totals(self) -> np.ndarray:
        """FP64 {mass, momentum, kinetic energy} over the fluid leaves, each level weighted by its
        volume in finest cells, 8^(L - l) (state.jl:333-356)."""
        out = (C.c_double * 5)()
        if self._tree is not None:
            check(lib().oal_q19_octree_totals(self._tree, out))
        else:
            check(lib().oal_q19_level_totals(self._h, out, None))
        return np.array(out[:])

    def total_mass(self) -> float:
        return float(self.totals()[0])

    def total_momentum(self) -> np.ndarray:
        return self.totals()[1:4]

    def kinetic_energy(self) -> float:
        return float(self.totals()[4])

    def device_state(self, level: int = 1):
        f, u, rho = C.c_void_p(), C.c_void_p(), C.c_void_p()
        steps = C.c_int64()
        check(lib().oal_q19_level_device_state(self._level_handle(level), C.byref(f), C.byref(u), C.byref(rho),
                                               C.byref(steps)))
        return f.value, u.value, rho.value, steps.value


def collide_cells(f, omega, sigma, pfd, F):
    """The collision alone on the GPU over n cells (torch CUDA tensors: f (n,19), omega (n), pfd (n,6),
    F (n,3)); returns (out, rho, u). A test hook of the known-answer checks."""
    import torch
    dt = f.dtype
    prec = capi.OAL_STORE_F64 if dt == torch.float64 else capi.OAL_STORE_F32
    n = f.shape[0]
    out = torch.empty_like(f)
    rho = torch.empty(n, dtype=dt, device=f.device)
    u = torch.empty(n, 3, dtype=dt, device=f.device)
    args = [t.contiguous() for t in (f, omega, pfd, F)]
    stream = torch.cuda.current_stream(f.device).cuda_stream
    check(lib().oal_q19_collide_cells(prec, n, args[0].data_ptr(), args[1].data_ptr(), float(sigma),
                                      args[2].data_ptr(), args[3].data_ptr(), out.data_ptr(), rho.data_ptr(),
                                      u.data_ptr(), C.c_void_p(stream)))
    torch.cuda.current_stream(f.device).synchronize()
    return out, rho, u


def level_bytes_per_cell(dtype, sgs: str = "wale", hrr_sigma: float = 0.98) -> int:
    """Algorithmic HBM bytes of one cell update: the 19 populations read and written, the velocity and
    density written, and, when the velocity gradient is used (SGS or HRR), the previous velocity read
    (and the previous density for HRR)."""
    es = np.dtype(dtype).itemsize
    grad = sgs != "none" or hrr_sigma != 1.0
    return es * (2 * 19 + 3 + 1 + ((3 + (1 if hrr_sigma != 1.0 else 0)) if grad else 0))


def benchmark_periodic_box(n: int = 256, steps: int = 100, warmup: int = 10, precision=np.float32,
                           sgs: str = "wale", hrr_sigma: float = 0.98, nu_lattice: float = 0.001):
    """Time `steps` level steps of an n^3 periodic box (a Taylor-Green start) with CUDA events on the
    launching stream. Returns a dict (MLUPS, ms per step, algorithmic GB/s)."""
    import math
    import torch
    box = PeriodicBox(n)
    st = State(box, test_case_config(box, nu_lattice=nu_lattice, precision=precision, sgs=sgs, hrr_sigma=hrr_sigma))
    k = 2 * math.pi / n
    st.initialise(lambda x, y, z: (1.0, 0.05 * np.sin(k * x) * np.cos(k * y), -0.05 * np.cos(k * x) * np.sin(k * y),
                                   0.0 * x))
    s = torch.cuda.Stream()
    st.advance(warmup, s)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    st.advance(steps, s)
    e1.record(s)
    s.synchronize()
    ms = e0.elapsed_time(e1) / steps
    cells = n ** 3
    ke = st.kinetic_energy()
    st.close()
    bpc = level_bytes_per_cell(precision, sgs, hrr_sigma)
    return {"workload": f"q19_periodic_{n}^3_{np.dtype(precision).name}_{sgs}_sigma{hrr_sigma:g}", "cells": cells,
            "steps": steps, "ms_per_step": round(ms, 4), "mlups": round(cells / ms / 1e3, 1),
            "bytes_per_cell": bpc, "achieved_gbs": round(cells * bpc / ms / 1e6, 1), "kinetic_energy": ke,
            "gpu_launches": steps}


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="Time the D3Q19 octree step on an n^3 periodic box")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--sgs", default="wale", choices=list(SGS_CODES))
    ap.add_argument("--sigma", type=float, default=0.98)
    ap.add_argument("--naca", action="store_true", help="the 3-level NACA 0012 case instead of the periodic box")
    a = ap.parse_args()
    dt = np.float32 if a.precision == "f32" else np.float64
    if a.naca:
        print(json.dumps(benchmark_naca(a.steps, a.warmup, dt)))
    else:
        print(json.dumps(benchmark_periodic_box(a.n, a.steps, a.warmup, dt, a.sgs, a.sigma)))



def naca4_symmetric_triangles(chord: float, thickness: float = 0.12, n_points: int = 200, aoa_deg: float = 0.0,
                              leading_edge=(0.0, 0.0), span=(0.0, 1.0)) -> np.ndarray:
    """Triangles of a symmetric NACA 4-digit section extruded along z over `span`: the standard
    thickness distribution y_t = 5 t c (0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 - 0.1036 x^4)
    (closed trailing edge), cosine spacing, rotated nose-up by `aoa_deg` about the quarter chord.
    End caps are closed; a span that covers a periodic axis has its caps dropped by the generator."""
    beta = np.linspace(0.0, np.pi, n_points)
    xc = 0.5 * (1 - np.cos(beta))
    yt = 5 * thickness * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc ** 2 + 0.2843 * xc ** 3 - 0.1036 * xc ** 4)
    # counter-clockwise contour: upper surface trailing edge -> leading edge, then the lower one back
    x = np.concatenate([xc[::-1], xc[1:-1]]) * chord
    y = np.concatenate([yt[::-1], -yt[1:-1]]) * chord
    a = np.radians(aoa_deg)
    xq = x - 0.25 * chord
    xr = np.cos(a) * xq + np.sin(a) * y + 0.25 * chord + leading_edge[0]
    yr = -np.sin(a) * xq + np.cos(a) * y + leading_edge[1]
    z0, z1 = span
    tri = []
    n = len(xr)
    for i in range(n):
        j = (i + 1) % n
        p0, p1 = (xr[i], yr[i]), (xr[j], yr[j])
        tri.append(((p0[0], p0[1], z0), (p1[0], p1[1], z0), (p1[0], p1[1], z1)))
        tri.append(((p0[0], p0[1], z0), (p1[0], p1[1], z1), (p0[0], p0[1], z1)))
    cx, cy = xr.mean(), yr.mean()
    for zc, flip in ((z0, True), (z1, False)):
        for i in range(n):
            j = (i + 1) % n
            t = ((cx, cy, zc), (xr[i], yr[i], zc), (xr[j], yr[j], zc))
            tri.append((t[0], t[2], t[1]) if flip else t)
    return np.array(tri, np.float64)


def naca_case(chord: int = 128, levels: int = 3, aoa_deg: float = 4.0, u_lattice: float = 0.04, reynolds: float = 1e5,
              domain=(1024.0, 512.0, 40.0), leading_edge_x: float = 320.0, precision=np.float32,
              band_fine: int = 8):
    """A NACA 0012 in a span-periodic box (x: inlet / outlet, y: slip, z: periodic), the surface band at
    the finest level, D3Q19 HRR (sigma 0.98) with WALE 0.5; lengths in finest cells (dx_finest = 1).
    Returns (mesh, config)."""
    tri = naca4_symmetric_triangles(chord, 0.12, 241, aoa_deg, (leading_edge_x, domain[1] / 2),
                                    (-8.0, domain[2] + 8.0))
    spec = MeshSpec(domain=domain, periodic=(False, False, True), levels=levels, dx_finest=1.0, band_fine=band_fine,
                    faces=("inlet", "outlet", "slip", "slip", "periodic", "periodic"))
    mesh = generate(tri, spec)
    nu = u_lattice * chord / reynolds
    cfg = CaseConfig(nu_lattice=nu, u_lattice=u_lattice, velocity=1.0, hrr_sigma=0.98, sgs="wale", c_wale=0.5,
                     precision=precision, dx=1.0)
    cfg.extra.update(chord=chord, aoa_deg=aoa_deg, reynolds=reynolds, span=domain[2])
    return mesh, cfg


def benchmark_naca(steps: int = 100, warmup: int = 20, precision=np.float32, **kw) -> dict:
    """Time `steps` coarse steps of the NACA 0012 case (CUDA events on the launching stream) after a
    uniform start and `warmup` steps; MLUPS counts the fluid cell updates of a coarse step over all
    levels, W = sum_l fluid_l 2^(l - 1) (run.jl:99). The forces are those of the last step, coarse-
    lattice units times 4^(L - 1) in finest units; after a short run they are a start transient."""
    import time
    import torch
    t0 = time.perf_counter()
    mesh, cfg = naca_case(precision=precision, **kw)
    t_mesh = time.perf_counter() - t0
    st = State(mesh, cfg)
    st.initialise_uniform(1.0, cfg.u_lattice, 0.0, 0.0)
    s = torch.cuda.Stream()
    st.advance(warmup, s)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    st.advance(steps - 1, s)
    st.advance(1, s, collect=True)
    e1.record(s)
    s.synchronize()
    ms = e0.elapsed_time(e1) / steps
    W = mesh.work_W()
    L = mesh.nlevels
    F = st.forces * 4.0 ** (L - 1)
    q = 0.5 * cfg.u_lattice ** 2 * cfg.extra["chord"] * cfg.extra["span"]
    mass = st.total_mass()
    st.close()
    bpc = level_bytes_per_cell(precision, "wale", 0.98)
    per = [(lv.level, lv.counts["fluid_total"]) for lv in mesh.levels]
    return {"workload": f"naca0012_c{cfg.extra['chord']}_aoa{cfg.extra['aoa_deg']:g}_re{cfg.extra['reynolds']:g}_"
                        f"{L}levels_{np.dtype(precision).name}_hrr0.98_wale0.5",
            "finest_equivalent_cells": int(np.prod(mesh.levels[-1].n)), "fluid_per_level": per, "work_W": W,
            "coarse_steps": steps, "ms_per_coarse_step": round(ms, 4), "mlups": round(W / ms / 1e3, 1),
            "bytes_per_cell_update": bpc, "achieved_gbs": round(W * bpc / ms / 1e6, 1),
            "mesh_seconds": round(t_mesh, 2), "cd_transient": float(F[0] / q), "cl_transient": float(F[1] / q),
            "mass": mass, "leak_cells": mesh.counts["leak_cells"]}


if __name__ == "__main__":
    main()


# ---- the mesh file (octree.jl:158-233) ---------------------------------------------------------
MESH_MAGIC = b"OCTQ19M\0"
MESH_FORMAT = 5


def _w_i64(buf, v):
    buf += np.array([v], "<i8").tobytes()


def _w_string(buf, s: str):
    b = s.encode()
    _w_i64(buf, len(b))
    buf += b


def _w_array(buf, a: np.ndarray, julia_dims):
    """_write_array: ndims, the dims in Julia's order, the elements in memory order (the C-order
    array whose shape is julia_dims reversed)."""
    _w_i64(buf, len(julia_dims))
    for d in julia_dims:
        _w_i64(buf, int(d))
    buf += np.ascontiguousarray(a).tobytes()


def _toml(counts: dict) -> str:
    """The generator's counts as TOML: integers, and per_level as an array of tables."""
    lines = [f"{k} = {int(v)}" for k, v in counts.items() if not isinstance(v, (list, dict))]
    for t in counts.get("per_level", []):
        lines.append("")
        lines.append("[[per_level]]")
        lines += [f"{k} = {int(v)}" for k, v in t.items()]
    return "\n".join(lines) + "\n"


def write_mesh(path, mesh: OctMesh, triangles=None, offset=(0.0, 0.0, 0.0), config_sha: str = "",
               stl_sha: str = "") -> str:
    """Write `mesh` as the reference's mesh file (write_mesh, octree.jl:172-204): magic, format,
    domain, offset, periodic axes, the two hashes, the counts (TOML), the placed triangles and every
    level's tables in Julia's element order, followed by the SHA-256 of all that. Returns the hex
    digest."""
    import hashlib
    spec = mesh.spec
    tri = np.zeros((0, 3, 3)) if triangles is None else np.asarray(triangles, np.float64).reshape(-1, 3, 3)
    buf = bytearray(MESH_MAGIC)
    _w_i64(buf, MESH_FORMAT)
    buf += np.asarray(spec.domain, "<f8").tobytes()
    buf += np.asarray(offset, "<f8").tobytes()
    buf += np.asarray([bool(p) for p in spec.periodic], np.uint8).tobytes()
    _w_string(buf, config_sha)
    _w_string(buf, stl_sha)
    _w_string(buf, _toml(mesh.counts))
    _w_i64(buf, tri.shape[0])
    _w_array(buf, tri.astype("<f8"), (3, 3, tri.shape[0]))
    _w_i64(buf, mesh.nlevels)
    for lv in mesh.levels:
        _w_i64(buf, lv.level)
        buf += np.array([lv.dx], "<f8").tobytes()
        for v in lv.n:
            _w_i64(buf, v)
        _w_i64(buf, lv.nocts)
        no = lv.nocts
        _w_array(buf, lv.origin.astype("<i4"), (3, no))
        _w_array(buf, (lv.real != 0).astype(np.uint8), (no,))
        _w_array(buf, lv.kind.astype(np.uint8), (8, no))
        _w_array(buf, lv.face.astype(np.uint8), (8, no))
        _w_array(buf, lv.onbr.astype("<i4"), (27, no))
        _w_array(buf, lv.cutidx.astype("<i4"), (8, no))
        _w_array(buf, lv.special.astype("<u4"), (8, no))
        for name, dt in (("cut_slot", "<i4"), ("cut_off", "<i4"), ("cut_dir", np.uint8), ("cut_q", "<f4"),
                         ("cut_tri", "<i4")):
            a = getattr(lv, name).astype(dt)
            _w_array(buf, a, (a.shape[0],))
        cp = (lv.cut_partner != 0).astype(np.uint8)
        _w_array(buf, cp, (cp.shape[0],))
        ng, nr = lv.ghost_slot.shape[0], lv.restrict_slot.shape[0]
        _w_array(buf, lv.ghost_slot.astype("<i4"), (ng,))
        _w_array(buf, lv.ghost_donor.astype("<i4"), (64, ng))
        _w_array(buf, lv.ghost_w.astype("<f4"), (64, ng))
        _w_array(buf, lv.restrict_slot.astype("<i4"), (nr,))
        _w_array(buf, lv.restrict_src.astype("<i4"), (64, nr))
        _w_array(buf, (lv.restrict_cubic != 0).astype(np.uint8), (nr,))
    digest = hashlib.sha256(bytes(buf)).digest()
    tmp = str(path) + ".tmp"
    with open(tmp, "wb") as io:
        io.write(bytes(buf))
        io.write(digest)
    os.replace(tmp, path)
    return digest.hex()


class _Reader:
    def __init__(self, data: bytes):
        self.d, self.o = data, 0

    def take(self, n: int) -> bytes:
        b = self.d[self.o:self.o + n]
        if len(b) != n:
            raise ValueError("mesh file ends early")
        self.o += n
        return b

    def i64(self) -> int:
        return int(np.frombuffer(self.take(8), "<i8")[0])

    def f64(self, n=1):
        return np.frombuffer(self.take(8 * n), "<f8").copy()

    def string(self) -> str:
        return self.take(self.i64()).decode()

    def array(self, dt):
        nd = self.i64()
        dims = [self.i64() for _ in range(nd)]
        n = int(np.prod(dims)) if dims else 1
        a = np.frombuffer(self.take(n * np.dtype(dt).itemsize), dt).copy()
        return a.reshape(tuple(reversed(dims)))


def read_mesh(path, faces=("periodic",) * 6) -> OctMesh:
    """Read a mesh file written by the reference's write_mesh or by write_mesh here (read_mesh,
    octree.jl:206-233): checks the SHA-256 trailer, the magic and the format. The domain-face
    conditions are not part of the file; `faces` names them (-x +x -y +y -z +z) as MeshSpec does.
    The triangles are returned as the mesh's `triangles` (ntri, 3, 3)."""
    import hashlib
    import tomllib
    data = open(path, "rb").read()
    if len(data) <= 32:
        raise ValueError(f"{path} is not a mesh file")
    if hashlib.sha256(data[:-32]).digest() != data[-32:]:
        raise ValueError(f"{path}: hash mismatch (the file is damaged or truncated)")
    r = _Reader(data[:-32])
    if r.take(len(MESH_MAGIC)) != MESH_MAGIC:
        raise ValueError(f"{path}: not an octree D3Q19 mesh")
    fmt = r.i64()
    if fmt != MESH_FORMAT:
        raise ValueError(f"{path}: mesh format {fmt}, expected {MESH_FORMAT}")
    domain = tuple(float(v) for v in r.f64(3))
    offset = tuple(float(v) for v in r.f64(3))
    periodic = tuple(bool(v) for v in np.frombuffer(r.take(3), np.uint8))
    config_sha, stl_sha = r.string(), r.string()
    counts = tomllib.loads(r.string())
    nt = r.i64()
    tri = r.array("<f8").reshape(nt, 3, 3)
    nl = r.i64()
    face_codes = [capi.Q19_FACE_NAMES[f] for f in faces]
    levels = []
    for _ in range(nl):
        level = r.i64()
        dx = float(r.f64(1)[0])
        n = tuple(r.i64() for _ in range(3))
        nocts = r.i64()
        arrays = {"origin": r.array("<i4"), "real": r.array(np.uint8), "kind": r.array(np.uint8),
                  "face": r.array(np.uint8), "onbr": r.array("<i4"), "cutidx": r.array("<i4"),
                  "special": r.array("<u4")}
        for name, dt in (("cut_slot", "<i4"), ("cut_off", "<i4"), ("cut_dir", np.uint8), ("cut_q", "<f4"),
                         ("cut_tri", "<i4"), ("cut_partner", np.uint8), ("ghost_slot", "<i4"),
                         ("ghost_donor", "<i4"), ("ghost_w", "<f4"), ("restrict_slot", "<i4"),
                         ("restrict_src", "<i4"), ("restrict_cubic", np.uint8)):
            arrays[name] = r.array(dt)
        arrays = {k: np.ascontiguousarray(v.astype(v.dtype.newbyteorder("="))) for k, v in arrays.items()}
        if arrays["onbr"].shape[0] != nocts:
            raise ValueError(f"{path}: level {level} holds {arrays['onbr'].shape[0]} octs, header says {nocts}")
        per = counts.get("per_level", [])
        m = Mesh(arrays, n, dx, face_codes, nt, per[level - 1] if level - 1 < len(per) else {})
        m.level = level
        m.domain = tuple(v * dx for v in n)
        levels.append(m)
    if r.o != len(r.d):
        raise ValueError(f"{path}: {len(r.d) - r.o} bytes after the last level")
    spec = MeshSpec(domain=domain, periodic=periodic, levels=nl, dx_finest=levels[-1].dx if levels else 1.0,
                    faces=tuple(faces))
    mesh = OctMesh(levels, {k: v for k, v in counts.items()}, spec)
    mesh.triangles = tri
    mesh.offset, mesh.config_sha, mesh.stl_sha = offset, config_sha, stl_sha
    return mesh


# ---------------------------------------------------------------- checkpoint
CHECKPOINT_MAGIC = b"OCTQ19C\0"
CHECKPOINT_FORMAT = 1


def _sha64(s: str) -> bytes:
    """A hash string as the checkpoint holds it: space-padded or cut to 64 bytes (rpad(s, 64)[1:64])."""
    b = s.encode()
    return (b + b" " * 64)[:64]


def pack_checkpoint(levels, precision, step: int, u_inlet: float, mass0: float, n_avg: int = 0, sums=None,
                    config_sha: str = "", stl_sha: str = "") -> bytes:
    """The checkpoint file of write_checkpoint! (io_run.jl:277-291), version 1: magic, version,
    sizeof(T), the config and STL hashes (64 bytes each), step, u_inlet, mass0, the force averages'
    count and nine sums, the level count, then per level the oct count and f, g, u, v, rho, rhob
    (both buffers, the current one first) and the wall-model friction velocities tau_w. `levels`:
    per level a dict of C-order arrays f (nocts, 19, 8), g, u (nocts, 3, 8), v, rho (nocts, 8),
    rhob, tau_w (ncut,), whose memory is the reference's column-major (8, 19, nocts) etc."""
    dt = np.dtype(precision).newbyteorder("<")
    if dt.itemsize not in (4, 8):
        raise ValueError("precision must be float32 or float64")
    sums = np.zeros(9) if sums is None else np.asarray(sums, np.float64).reshape(9)
    out = bytearray(CHECKPOINT_MAGIC)
    out += np.array([CHECKPOINT_FORMAT, dt.itemsize], "<i8").tobytes()
    out += _sha64(config_sha) + _sha64(stl_sha)
    out += np.array([step], "<i8").tobytes() + np.array([u_inlet, mass0], "<f8").tobytes()
    out += np.array([n_avg], "<i8").tobytes() + sums.astype("<f8").tobytes()
    out += np.array([len(levels)], "<i8").tobytes()
    for lv in levels:
        no = int(lv["f"].shape[0])
        shapes = {"f": (no, 19, 8), "g": (no, 19, 8), "u": (no, 3, 8), "v": (no, 3, 8), "rho": (no, 8), "rhob": (no, 8)}
        out += np.array([no], "<i8").tobytes()
        for name in ("f", "g", "u", "v", "rho", "rhob"):
            a = np.asarray(lv[name])
            if a.shape != shapes[name]:
                raise ValueError(f"checkpoint array {name}: shape {a.shape}, expected {shapes[name]}")
            out += np.ascontiguousarray(a, dt).tobytes()
        tw = np.asarray(lv.get("tau_w", np.zeros(0)))
        out += np.array([tw.size], "<i8").tobytes() + np.ascontiguousarray(tw, dt).tobytes()
    return bytes(out)


def unpack_checkpoint(data: bytes, precision=None, config_sha: str | None = None, stl_sha: str | None = None,
                      octs=None, ncut=None) -> dict:
    """Parse a checkpoint (read_checkpoint!, io_run.jl:294-314) with the reference's checks: the
    magic, the version, the precision (when given), the case hashes (when given; compared after
    stripping the padding), the level count and each level's oct count and tau_w size (when
    given), and no trailing data. Returns the header fields and the per-level arrays."""
    r = _Reader(data)

    def fail(msg):
        raise ValueError(msg)

    try:
        if r.take(len(CHECKPOINT_MAGIC)) != CHECKPOINT_MAGIC:
            fail("not a checkpoint")
        if r.i64() != CHECKPOINT_FORMAT:
            fail("checkpoint format")
        size = r.i64()
        if size not in (4, 8) or (precision is not None and size != np.dtype(precision).itemsize):
            fail("checkpoint precision differs from the run's")
        dt = np.dtype("<f4" if size == 4 else "<f8")
        csha, ssha = r.take(64).decode().strip(), r.take(64).decode().strip()
        if (config_sha is not None and csha != config_sha) or (stl_sha is not None and ssha != stl_sha):
            fail("checkpoint belongs to another case (config or STL hash differs)")
        step = r.i64()
        u_inlet, mass0 = (float(v) for v in r.f64(2))
        n_avg = r.i64()
        sums = r.f64(9)
        nl = r.i64()
        if octs is not None and nl != len(octs):
            fail("checkpoint level count differs")
        levels = []
        for l in range(nl):
            no = r.i64()
            if octs is not None and no != octs[l]:
                fail("checkpoint oct count differs")
            lv = {}
            for name, shape in (("f", (no, 19, 8)), ("g", (no, 19, 8)), ("u", (no, 3, 8)), ("v", (no, 3, 8)),
                                ("rho", (no, 8)), ("rhob", (no, 8))):
                n = int(np.prod(shape))
                lv[name] = np.frombuffer(r.take(n * size), dt).reshape(shape).astype(dt.newbyteorder("="))
            nw = r.i64()
            if ncut is not None and nw != ncut[l]:
                fail("checkpoint wall-model size differs")
            lv["tau_w"] = np.frombuffer(r.take(nw * size), dt).astype(dt.newbyteorder("="))
            levels.append(lv)
    except ValueError as e:
        if str(e) == "mesh file ends early":
            raise ValueError("checkpoint ends early") from None
        raise
    if r.o != len(r.d):
        raise ValueError("checkpoint has unexpected trailing data")
    return dict(precision=dt.newbyteorder("="), config_sha=csha, stl_sha=ssha, step=step, u_inlet=u_inlet,
                mass0=mass0, n_avg=n_avg, sums=sums, levels=levels)


def _level_ncut(m) -> int:
    cs = getattr(m, "cut_slot", None)
    return 0 if cs is None else int(cs.shape[0])


def write_checkpoint(st: "State", out, n_avg: int = 0, sums=None, keep: int = 2) -> str:
    """write_checkpoint! (io_run.jl:277-291): `out`/checkpoints/checkpoint_<step, 9 digits>.bin,
    written to a .tmp file and renamed; keeps the newest `keep`. Both buffers of every level are
    written (the current one first; a refined mesh's ghost fill blends the previous one). tau_w is
    zero (the octree wall model is not built here)."""
    d = os.path.join(str(out), "checkpoints")
    os.makedirs(d, exist_ok=True)
    levels = []
    for l, m in enumerate(st.level_meshes, start=1):
        f, u, rho = st.buffer(0, l)
        g, v, rhob = st.buffer(1, l)
        levels.append(dict(f=f, g=g, u=u, v=v, rho=rho, rhob=rhob, tau_w=np.zeros(_level_ncut(m), st.dtype)))
    data = pack_checkpoint(levels, st.dtype, st.step, float(st.cfg.u_lattice), float(st.mass0), n_avg, sums,
                           st.config_sha, st.stl_sha)
    path = os.path.join(d, f"checkpoint_{st.step:09d}.bin")
    with open(path + ".tmp", "wb") as io:
        io.write(data)
    os.replace(path + ".tmp", path)
    files = sorted(f for f in os.listdir(d) if f.startswith("checkpoint_") and f.endswith(".bin"))
    for f in files[:max(0, len(files) - keep)]:
        os.remove(os.path.join(d, f))
    return path


def read_checkpoint(st: "State", path) -> dict:
    """read_checkpoint! (io_run.jl:294-314): the case and precision must match the state; restores
    both buffers of every level, the step and mass0. Returns the header (with n_avg and the nine
    force sums for the caller's histories)."""
    with open(path, "rb") as io:
        data = io.read()
    ck = unpack_checkpoint(data, st.dtype, st.config_sha, st.stl_sha, [m.nocts for m in st.level_meshes],
                           [_level_ncut(m) for m in st.level_meshes])
    for l, lv in enumerate(ck["levels"], start=1):
        st.set_buffer(0, lv["f"], lv["u"], lv["rho"], l)
        st.set_buffer(1, lv["g"], lv["v"], lv["rhob"], l)
    st.step = ck["step"]
    st.mass0 = ck["mass0"]
    return ck


def resume_checkpoint(st: "State", out):
    """resume_checkpoint! (io_run.jl:317-323): restore the latest checkpoint under `out`; returns
    its step, or None when there is none."""
    d = os.path.join(str(out), "checkpoints")
    if not os.path.isdir(d):
        return None
    files = sorted(f for f in os.listdir(d) if f.startswith("checkpoint_") and f.endswith(".bin"))
    if not files:
        return None
    return read_checkpoint(st, os.path.join(d, files[-1]))["step"]
