"""CPU ORACLE — test infrastructure only.

C++ restatements of the reference's D3Q27 cumulant level step (oal_oracle.cpp), of its D3Q19
octree level step (oal_oracle_q19.cpp) and of its D3Q39 entropic KBC level step
(oal_oracle_q39.cpp); each source holds the file:line map into the reference.
Only tests/, the smoke check and the CPU-baseline leg of bench.py use it; the product path never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboal_oracle.so"

_lib = None


def build(force: bool = False) -> Path:
    deps = [HERE / "oal_oracle.cpp", HERE / "oal_oracle_q19.cpp", HERE / "oal_oracle_q39.cpp", HERE / "oal_oracle_surface.cpp",
            HERE.parent / "include" / "oal.h", HERE.parent / "openaerolab_alpha_01_b200" / "csrc" / "kbc_math.h"]
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "liboal_oracle.so"], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        i32 = C.c_int32
        L.ora_d3q27_tables.argtypes = [vp] * 7
        L.ora_default_step_params.argtypes = [vp]
        L.ora_surface_map.argtypes = [i32, vp, vp, vp, C.c_int64, vp, vp, i32, i32, i32, i32, i32] + [C.c_float] * 6 + [vp, vp, vp]
        L.ora_build_box.argtypes = [i32, i32, i32, i32, vp, vp]
        L.ora_sphere.argtypes = [i32, vp, C.c_double, C.c_double, C.c_double, C.c_double, vp]
        L.ora_sphere.restype = C.c_int64
        L.ora_init_feq_f64.argtypes = [i32, vp, vp, i32, vp]
        for n in ("ora_step_d3q27_f64", "ora_step_d3q27_f32"):
            getattr(L, n).argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
            getattr(L, n).restype = C.c_int
        L.ora_mass_momentum_f64.argtypes = [i32, vp, vp, vp]
        for n in ("ora_step_d3q27_pi_f64", "ora_step_d3q27_pi_f32"):
            getattr(L, n).argtypes = [i32, i32, i32, i32] + [vp] * 14
            getattr(L, n).restype = C.c_int
        L.ora_pi_neq_f64.argtypes = [i32, vp, vp, vp, vp, i32, vp]
        for n in ("ora_svv_d3q27_f64", "ora_svv_d3q27_f32"):
            getattr(L, n).argtypes = [i32, vp, vp, C.c_float, C.c_float, vp, vp, vp]
        for n in ("ora_nscbc_outlet_f64", "ora_nscbc_outlet_f32"):
            getattr(L, n).argtypes = [i32, i32, i32, i32, vp, vp, i32, C.c_float, C.c_float, C.c_float, vp, vp, vp]
        L.ora_q19_tables.argtypes = [vp] * 6
        L.ora_q19_periodic_box.argtypes = [i32, i32, i32, vp, vp]
        L.ora_q19_periodic_box.restype = C.c_int
        i64 = C.c_int64
        L.ora_q19_collide_f32.argtypes = [i64, vp, vp, C.c_float, vp, vp, vp, vp, vp]
        L.ora_q19_collide_f64.argtypes = [i64, vp, vp, C.c_double, vp, vp, vp, vp, vp]
        L.ora_q19_reference_collide_f32.argtypes = [i64, vp, vp, C.c_float, vp, vp, vp]
        L.ora_q19_reference_collide_f64.argtypes = [i64, vp, vp, C.c_double, vp, vp, vp]
        for suf in ("f32", "f64"):
            getattr(L, f"ora_q19_step_{suf}").argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, vp]
            getattr(L, f"ora_q19_step_walls_{suf}").argtypes = [vp] * 9
            getattr(L, f"ora_q19_initialise_{suf}").argtypes = [i64, vp, vp, vp, vp, C.c_double, vp, vp, vp]
        L.ora_q19_forces.argtypes = [vp, vp, vp, vp]
        for suf in ("f32", "f64"):
            getattr(L, f"ora_q19_fill_{suf}").argtypes = [vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp, vp]
            getattr(L, f"ora_q19_restrict_{suf}").argtypes = [vp, vp, C.c_double, C.c_double, vp, vp, vp]
        for suf in ("f64", "f32"):
            getattr(L, f"ora_step_d3q27_refined_{suf}").argtypes = (
                [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, i32, i32, i32, vp, vp, vp, vp, vp,
                 vp, C.c_double, C.c_double, i32])
            getattr(L, f"ora_step_d3q27_refined_{suf}").restype = C.c_int
            getattr(L, f"ora_restrict_d3q27_{suf}").argtypes = (
                [i32, vp, vp, vp, vp, i32, vp, i32, i32, i32, vp, vp, C.c_double, C.c_double, i32, i32])
        for suf in ("f64", "f32"):
            getattr(L, f"ora_bouzidi_linear_{suf}").argtypes = [i32, vp, vp, i32, vp, vp, C.c_float, i32, C.c_float,
                                                                 C.c_float, vp, vp]
            getattr(L, f"ora_bouzidi_linear_{suf}").restype = C.c_int
        L.ora_q39_tables.argtypes = [vp] * 5
        L.ora_q39_exp.argtypes = [i64, vp, vp]
        L.ora_q39_log.argtypes = [i64, vp, vp]
        L.ora_q39_equilibrium.argtypes = [i64, vp, vp, vp, vp]
        L.ora_q39_inlet_equilibrium.argtypes = [C.c_float, vp]
        L.ora_q39_collide_cells.argtypes = [i64, vp, vp, vp, vp, vp, vp, vp]
        L.ora_q39_step.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, vp]
        L.ora_q39_step_ex.argtypes = [i32, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def d3q27_tables():
    cx, cy, cz, opp, my, mz = (np.zeros(27, np.int32) for _ in range(6))
    w = np.zeros(27)
    lib().ora_d3q27_tables(_p(cx), _p(cy), _p(cz), _p(w), _p(opp), _p(my), _p(mz))
    return dict(cx=cx, cy=cy, cz=cz, w=w, opp=opp, mirror_y=my, mirror_z=mz)


def build_box(bx, by, bz, periodic_mask):
    n = bx * by * bz
    coords = np.zeros((n, 3), np.int32)
    nbr = np.zeros((27, n), np.int32)
    lib().ora_build_box(bx, by, bz, periodic_mask, _p(coords), _p(nbr))
    return coords, nbr


def sphere(coords, centre, radius):
    nb = coords.shape[0]
    obst = np.zeros((nb, 512), np.uint8)
    n = lib().ora_sphere(nb, _p(np.ascontiguousarray(coords, np.int32)), *map(float, centre), float(radius), _p(obst))
    return obst, int(n)


def default_step_params(**overrides):
    """oal_step_params with the reference's configuration defaults, filled by the oracle library
    (the struct type is the product's ctypes mirror of include/oal.h; no product code is loaded)."""
    from openaerolab_alpha_01_b200._capi import StepParams
    p = StepParams()
    lib().ora_default_step_params(C.addressof(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


class OracleCase:
    """A case built by the oracle alone: coords, neighbour table, obstacle, shape, initial fields
    and the step parameters."""

    def __init__(self, coords, nbr, shape, obstacle, rho, vel, params, meta):
        self.coords, self.nbr, self.shape, self.obstacle = coords, nbr, shape, obstacle
        self.rho, self.vel, self.params, self.meta = rho, vel, params, meta

    @property
    def n_blocks(self):
        return int(self.coords.shape[0])

    def level(self, dtype=np.float32):
        L = OracleLevel(self.coords, self.nbr, self.shape, obstacle=self.obstacle, dtype=dtype)
        L.init_equilibrium(self.rho, self.vel)
        return L


def sphere_channel(nx=256, ny=128, nz=128, diameter=24.0, centre_x=64.0, u_inlet=0.05, re=1000.0, c_wale=0.2):
    """The sphere channel (inlet at x_min, zero-gradient outlet, lateral mirrors, analytic sphere with
    half-way walls and the drag collected) from the oracle's own block builder and sphere mask."""
    coords, nbr = build_box(nx // 8, ny // 8, nz // 8, 0)
    obst, n_solid = sphere(coords, (centre_x, ny / 2.0, nz / 2.0), diameter / 2.0)
    nb = coords.shape[0]
    rho = np.ones((nb, 512))
    vel = np.zeros((3, nb, 512))
    vel[0] = np.where(obst != 0, 0.0, u_inlet)
    nu = u_inlet * diameter / re
    p = default_step_params(tau=3.0 * nu + 0.5, c_wale=c_wale, u_inlet=u_inlet, solid_bc=1, collect_forces=1)
    return OracleCase(coords, nbr, (nx, ny, nz), obst, rho, vel, p, dict(n_solid=n_solid, nu=nu))


def surface_map(tri, rho, vel, obstacle, ptr, dims, radius=8, recover=1, tau=0.6, c_wale=0.2, nu_bg=0.0,
                pscale=1.0, sscale=1.0, moment_center=(0.0, 0.0, 0.0), cs2=1.0 / 3.0):
    """Surface-stress mapping (src/forces/surface.jl:636-1331) on host fields in the reference
    layout (rho (nb, 512), vel (3, nb, 512), obstacle (nb, 512)); ptr: 1-based block pointer over
    the dims block grid, x fastest. Returns (per-triangle (n, 6) float32, per-triangle force and
    moment (n, 9) float64)."""
    tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 7)
    n = tri.shape[0]
    rho = np.ascontiguousarray(rho, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    obst = np.ascontiguousarray(obstacle if obstacle is not None else np.zeros(rho.shape, np.uint8), np.uint8)
    ptr = np.ascontiguousarray(ptr, np.int32)
    mc = np.ascontiguousarray(moment_center, np.float32)
    out = np.zeros((n, 6), np.float32)
    part = np.zeros((n, 9))
    lib().ora_surface_map(n, _p(tri), _p(rho), _p(vel), int(rho.size), _p(obst), _p(ptr), *map(int, dims), int(radius),
                          int(recover), tau, c_wale, nu_bg, pscale, sscale, cs2, _p(mc), _p(out), _p(part))
    return out, part


def init_feq(rho, vel, compressible=0):
    nb = rho.shape[0]
    f = np.zeros((27, nb, 512))
    lib().ora_init_feq_f64(nb, _p(np.ascontiguousarray(rho, np.float64)), _p(np.ascontiguousarray(vel, np.float64)),
                           compressible, _p(f))
    return f


def svv_d3q27(nb, nbr, obstacle, eps_x, eps_yz, f_in, f_out, f_post2=None):
    """The spectral vanishing viscosity post-pass (apply_svv_d3q19_postcollision!,
    kernel_svv_yz_d3q39.jl:426-458) on reference-layout arrays (27, nb, 512): f_out filtered in
    place from f_in; f_post2 (or None) receives the same values."""
    fn = lib().ora_svv_d3q27_f64 if f_out.dtype == np.float64 else lib().ora_svv_d3q27_f32
    fn(int(nb), _p(nbr), _p(obstacle), float(eps_x), float(eps_yz), _p(f_in), _p(f_out), _p(f_post2))


def _svv_on(params):
    return params.svv_x_epsilon > 0 or params.svv_yz_epsilon > 0


class OracleLevel:
    """Reference-layout state stepped by the CPU restatement (double or float)."""

    def __init__(self, coords, nbr, shape, obstacle=None, sponge=None, wall_dist=None, dtype=np.float64):
        self.coords = np.ascontiguousarray(coords, np.int32)
        self.nbr = np.ascontiguousarray(nbr, np.int32)
        self.nb = self.coords.shape[0]
        self.shape = tuple(int(s) for s in shape)
        self.obstacle = None if obstacle is None else np.ascontiguousarray(obstacle, np.uint8)
        self.sponge = None if sponge is None else np.ascontiguousarray(sponge, np.float32)
        self.wall_dist = None if wall_dist is None else np.ascontiguousarray(wall_dist, np.float32)
        self.dtype = np.dtype(dtype)
        nb = self.nb
        self.f = np.zeros((27, nb, 512), self.dtype)
        self.g = np.zeros_like(self.f)
        self.rho = np.ones((nb, 512), self.dtype)
        self.vel = np.zeros((3, nb, 512), self.dtype)
        self.vel_new = np.zeros_like(self.vel)
        self.pi_neq = np.zeros((6, nb, 512), self.dtype)
        self.force = np.zeros(3)

    def init_equilibrium(self, rho, vel, compressible=0):
        self.f[...] = init_feq(rho, vel, compressible).astype(self.dtype)
        self.rho[...] = rho
        self.vel[...] = vel
        self.pi_neq[...] = 0

    def step(self, params):
        force = np.zeros(3)
        if params.variable_nu_sgs:
            # variable nu_sgs: Pi_neq carried from step to step (kernel_cumulant.jl:546-588)
            fn = lib().ora_step_d3q27_pi_f64 if self.dtype == np.float64 else lib().ora_step_d3q27_pi_f32
            rc = fn(self.nb, *self.shape, _p(self.coords), _p(self.nbr), _p(self.obstacle), _p(self.sponge),
                    _p(self.wall_dist), C.addressof(params), _p(self.f), _p(self.g), None, _p(self.rho),
                    _p(self.vel_new), _p(self.vel), _p(self.pi_neq), _p(force))
        else:
            fn = lib().ora_step_d3q27_f64 if self.dtype == np.float64 else lib().ora_step_d3q27_f32
            rc = fn(self.nb, *self.shape, _p(self.coords), _p(self.nbr), _p(self.obstacle), _p(self.sponge),
                    _p(self.wall_dist), C.addressof(params), _p(self.f), _p(self.g), None, _p(self.rho),
                    _p(self.vel_new), _p(self.vel), _p(force))
        assert rc == 0
        if _svv_on(params):
            # the filter after the step kernels (timestep.jl:1576-1611)
            svv_d3q27(self.nb, self.nbr, self.obstacle, params.svv_x_epsilon, params.svv_yz_epsilon, self.f, self.g)
        self.f, self.g = self.g, self.f
        self.vel, self.vel_new = self.vel_new, self.vel
        if params.collect_forces:
            self.force = force
        if _svv_on(params) and params.variable_nu_sgs == 1:
            # the filter rewrote the populations after the refresh: Pi_neq of the filtered state
            self.pi_neq[...] = self.state_pi_neq(params.compressible_corr)
        return self

    def step_bouzidi(self, params, bz):
        """One step followed by the linear Bouzidi correction (timestep.jl:1752-1768): `bz` holds
        cells (n, 4) int32 (block, x, y, z) 1-based, q (n, 27) float16, q_min, ff_fallback,
        rel_cap, abs_cap."""
        p = type(params).from_buffer_copy(params)
        p.store_post_collision = 1
        post = np.zeros_like(self.f)
        force = np.zeros(3)
        if p.variable_nu_sgs:
            fn = lib().ora_step_d3q27_pi_f64 if self.dtype == np.float64 else lib().ora_step_d3q27_pi_f32
            rc = fn(self.nb, *self.shape, _p(self.coords), _p(self.nbr), _p(self.obstacle), _p(self.sponge),
                    _p(self.wall_dist), C.addressof(p), _p(self.f), _p(self.g), _p(post), _p(self.rho),
                    _p(self.vel_new), _p(self.vel), _p(self.pi_neq), _p(force))
        else:
            fn = lib().ora_step_d3q27_f64 if self.dtype == np.float64 else lib().ora_step_d3q27_f32
            rc = fn(self.nb, *self.shape, _p(self.coords), _p(self.nbr), _p(self.obstacle), _p(self.sponge),
                    _p(self.wall_dist), C.addressof(p), _p(self.f), _p(self.g), _p(post), _p(self.rho),
                    _p(self.vel_new), _p(self.vel), _p(force))
        assert rc == 0
        if _svv_on(p):
            svv_d3q27(self.nb, self.nbr, self.obstacle, p.svv_x_epsilon, p.svv_yz_epsilon, self.f, self.g, post)
        cells = np.ascontiguousarray(bz["cells"], np.int32)
        q = np.ascontiguousarray(np.asarray(bz["q"], np.float16).astype(np.float32))
        fb = lib().ora_bouzidi_linear_f64 if self.dtype == np.float64 else lib().ora_bouzidi_linear_f32
        rc = fb(self.nb, _p(self.nbr), _p(self.obstacle), int(cells.shape[0]), _p(cells), _p(q),
                bz.get("q_min", 0.001), int(bz.get("ff_fallback", 0)), bz.get("rel_cap", 0.0),
                bz.get("abs_cap", 0.0), _p(post), _p(self.g))
        assert rc == 0
        self.f, self.g = self.g, self.f
        self.vel, self.vel_new = self.vel_new, self.vel
        if p.variable_nu_sgs == 1:
            # the correction rewrote populations after the refresh: refresh again from the
            # corrected state (timestep.jl:1818-1834)
            self.pi_neq[...] = self.state_pi_neq(p.compressible_corr)
        return self

    def nscbc(self, all_blocks=False, p_target=1.0, sigma_relax=0.27, neq_blend=0.5):
        """The characteristic outlet on the current state (apply_nscbc_outlet_kernel!,
        kernel_nscbc_outlet.jl:80-340), athermal."""
        fn = lib().ora_nscbc_outlet_f64 if self.dtype == np.float64 else lib().ora_nscbc_outlet_f32
        fn(self.nb, *self.shape, _p(self.coords), _p(self.obstacle), int(bool(all_blocks)), p_target, sigma_relax,
           neq_blend, _p(self.f), _p(self.rho), _p(self.vel))
        return self

    def state_pi_neq(self, compressible=0):
        """Pi_neq of the stored state (compute_pi_neq_kernel!, kernel_pi_neq.jl:39-180): (6, nb, 512)
        in the order xx, yy, zz, xy, xz, yz, zero in solid cells."""
        out = np.zeros((6, self.nb, 512))
        c = lambda a: np.ascontiguousarray(a, np.float64)
        lib().ora_pi_neq_f64(self.nb, _p(self.obstacle), _p(c(self.f)), _p(c(self.rho)), _p(c(self.vel)),
                             int(compressible), _p(out))
        return out

    def mass_momentum(self):
        out = np.zeros(4)
        f = np.ascontiguousarray(self.f, np.float64)
        lib().ora_mass_momentum_f64(self.nb, _p(self.obstacle), _p(f), _p(out))
        return out


class OracleAMR:
    """recursive_step! (src/solver/solver_control.jl:55-560, default flags) over D3Q27 levels held
    in the reference layout: level 0 steps once per coarse step; every finer level steps twice per
    step of its parent (temporal weights 0 and 1/2 against the parent's state before and after its
    step), then is restricted onto the parent. `domains`: objects with coords (n,3), neighbor_table
    (27,n), obstacle (n,512) or None, bx_max/by_max/bz_max and shape (the level's cell extent)."""

    def __init__(self, domains, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.levels = []
        for d in domains:
            nb = d.coords.shape[0]
            dims = (int(d.bx_max), int(d.by_max), int(d.bz_max))
            ptr = np.zeros(dims[0] * dims[1] * dims[2], np.int32)
            for i, (bx, by, bz) in enumerate(np.asarray(d.coords).tolist()):
                ptr[(bx - 1) + dims[0] * ((by - 1) + dims[1] * (bz - 1))] = i + 1
            self.levels.append(dict(
                nb=nb, dims=dims, shape=tuple(int(v) for v in d.shape), ptr=ptr,
                coords=np.ascontiguousarray(d.coords, np.int32), nbr=np.ascontiguousarray(d.neighbor_table, np.int32),
                obstacle=None if d.obstacle is None else np.ascontiguousarray(d.obstacle, np.uint8),
                f=[np.zeros((27, nb, 512), self.dtype), np.zeros((27, nb, 512), self.dtype)],
                vel=[np.zeros((3, nb, 512), self.dtype), np.zeros((3, nb, 512), self.dtype)],
                rho=np.ones((nb, 512), self.dtype), parity=0, f_old=None, rho_old=None, vel_old=None, bz=None))

    def set_bouzidi(self, l, bz):
        """Linear Bouzidi cells of level l (the dict of OracleLevel.step_bouzidi), applied after each of
        its steps (timestep.jl:1752-1768), before the restriction onto its parent."""
        self.levels[l]["bz"] = bz

    def init_equilibrium(self, l, rho, vel, compressible=0):
        L = self.levels[l]
        L["f"][0][...] = init_feq(rho, vel, compressible).astype(self.dtype)
        L["rho"][...] = rho
        L["vel"][0][...] = vel
        L["parity"] = 0

    def state(self, l):
        L = self.levels[l]
        return L["f"][L["parity"]], L["rho"], L["vel"][L["parity"]]

    def _suf(self):
        return "f64" if self.dtype == np.float64 else "f32"

    def _step(self, l, params, t_sub, tw):
        L = self.levels[l]
        p = L["parity"]
        f_in, f_out = L["f"][p], L["f"][p ^ 1]
        v_in, v_out = L["vel"][p], L["vel"][p ^ 1]
        has_children = l + 1 < len(self.levels)
        if has_children:
            L["f_old"], L["rho_old"], L["vel_old"] = f_in.copy(), L["rho"].copy(), v_in.copy()
        P = params[l]
        seed = P.time_step_seed
        P.time_step_seed = seed + t_sub
        force = np.zeros(3)
        nx, ny, nz = L["shape"]
        if l == 0:
            fn = getattr(lib(), f"ora_step_d3q27_{self._suf()}")
            rc = fn(L["nb"], nx, ny, nz, _p(L["coords"]), _p(L["nbr"]), _p(L["obstacle"]), None, None,
                    C.addressof(P), _p(f_in), _p(f_out), None, _p(L["rho"]), _p(v_out), _p(v_in), _p(force))
        else:
            Pa = self.levels[l - 1]
            pp = Pa["parity"]
            fn = getattr(lib(), f"ora_step_d3q27_refined_{self._suf()}")
            rc = fn(L["nb"], nx, ny, nz, _p(L["coords"]), _p(L["nbr"]), _p(L["obstacle"]), C.addressof(P),
                    _p(f_in), _p(f_out), _p(L["rho"]), _p(v_out), _p(v_in), _p(force), Pa["nb"], _p(Pa["ptr"]),
                    *Pa["dims"], _p(Pa["f"][pp]), _p(Pa["rho"]), _p(Pa["vel"][pp]), _p(Pa["f_old"]),
                    _p(Pa["rho_old"]), _p(Pa["vel_old"]), float(params[l - 1].tau), float(tw), 1)
        P.time_step_seed = seed
        assert rc == 0
        if _svv_on(P):
            svv_d3q27(L["nb"], L["nbr"], L["obstacle"], P.svv_x_epsilon, P.svv_yz_epsilon, f_in, f_out)
        bz = L["bz"]
        if bz is not None and P.solid_bc == 3:
            post = f_out.copy()  # the step stores the post-collision populations as its output
            cells = np.ascontiguousarray(bz["cells"], np.int32)
            qf = np.ascontiguousarray(np.asarray(bz["q"], np.float16).astype(np.float32))
            fb = getattr(lib(), f"ora_bouzidi_linear_{self._suf()}")
            assert fb(L["nb"], _p(L["nbr"]), _p(L["obstacle"]), int(cells.shape[0]), _p(cells), _p(qf),
                      bz.get("q_min", 0.001), int(bz.get("ff_fallback", 0)), bz.get("rel_cap", 0.0),
                      bz.get("abs_cap", 0.0), _p(post), _p(f_out)) == 0
        L["parity"] ^= 1
        if has_children:
            self._step(l + 1, params, 2 * t_sub, 0.0)
            self._step(l + 1, params, 2 * t_sub + 1, 0.5)
            Ch = self.levels[l + 1]
            q = L["parity"]
            fn = getattr(lib(), f"ora_restrict_d3q27_{self._suf()}")
            fn(L["nb"], _p(L["coords"]), _p(L["f"][q]), _p(L["rho"]), _p(L["vel"][q]), Ch["nb"], _p(Ch["ptr"]),
               *Ch["dims"], _p(Ch["obstacle"]), _p(Ch["f"][Ch["parity"]]), float(params[l].tau),
               float(params[l + 1].tau), int(params[l].compressible_corr), int(params[l].level_visc_physical))

    def advance(self, params, n):
        for i in range(n):
            self._step(0, params, i, 0.0)
        return self


# ---- D3Q19 octree (oal_oracle_q19.cpp) ---------------------------------------------------------

def _suffix(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def q19_tables():
    cx, cy, cz = (np.zeros(19, np.int32) for _ in range(3))
    w = np.zeros(19)
    off, child = np.zeros((8, 19), np.int32), np.zeros((8, 19), np.int32)
    lib().ora_q19_tables(_p(cx), _p(cy), _p(cz), _p(w), _p(off), _p(child))
    return dict(cx=cx, cy=cy, cz=cz, w=w, src_off=off, src_child=child)


def q19_periodic_box(n0, n1, n2):
    """(origin (nocts, 3), onbr (nocts, 27) 1-based): level 1 of a periodic box, Morton order."""
    no = (n0 // 2) * (n1 // 2) * (n2 // 2)
    origin = np.zeros((no, 3), np.int32)
    onbr = np.zeros((no, 27), np.int32)
    assert lib().ora_q19_periodic_box(n0, n1, n2, _p(origin), _p(onbr)) == 0
    return origin, onbr


def q19_collide(f, omega, sigma, pfd, F, reference=False):
    """Closed-form collision (or, with reference=True, the per-direction form) of n cells."""
    dt = np.dtype(f.dtype)
    f = np.ascontiguousarray(f)
    n = f.shape[0]
    omega = np.ascontiguousarray(omega, dt)
    pfd = np.ascontiguousarray(pfd, dt)
    F = np.ascontiguousarray(F, dt)
    out = np.zeros((n, 19), dt)
    if reference:
        getattr(lib(), f"ora_q19_reference_collide_{_suffix(dt)}")(n, _p(f), _p(omega), sigma, _p(pfd), _p(F), _p(out))
        return out
    rho, u = np.zeros(n, dt), np.zeros((n, 3), dt)
    getattr(lib(), f"ora_q19_collide_{_suffix(dt)}")(n, _p(f), _p(omega), sigma, _p(pfd), _p(F), _p(out), _p(rho), _p(u))
    return out, rho, u


class OracleQ19Level:
    """One octree level stepped by the CPU restatement; arrays in the reference's layout (numpy
    C-order shapes: f (nocts, 19, 8), u (nocts, 3, 8), rho (nocts, 8)). `desc` (a level descriptor
    with its arrays kept alive by the caller) selects the step with domain faces and cut links."""

    def __init__(self, onbr, dtype=np.float32, desc=None):
        self.onbr = np.ascontiguousarray(onbr, np.int32)
        self.nocts = self.onbr.shape[0]
        self.dtype = np.dtype(dtype)
        self.desc = desc
        self.kind = None
        if desc is not None and desc.kind:
            self.kind = np.ctypeslib.as_array((C.c_uint8 * (8 * self.nocts)).from_address(desc.kind)).copy()
        self.mom = np.zeros(max(desc.nlinks, 1) if desc is not None else 1)
        self.forces = np.zeros(3)
        self.per_tri = None
        no = self.nocts
        self.f = np.zeros((no, 19, 8), self.dtype)
        self.g = np.zeros_like(self.f)
        self.u = np.zeros((no, 3, 8), self.dtype)
        self.v = np.zeros_like(self.u)
        self.rho = np.ones((no, 8), self.dtype)
        self.rhob = np.ones_like(self.rho)

    def initialise(self, params, rho, u, du=None):
        rho = np.ascontiguousarray(rho, self.dtype)
        u = np.ascontiguousarray(u, self.dtype)
        du = None if du is None else np.ascontiguousarray(du, self.dtype)
        getattr(lib(), f"ora_q19_initialise_{_suffix(self.dtype)}")(self.nocts * 8, _p(self.kind), _p(rho), _p(u),
                                                                    _p(du), float(params.nu), _p(self.f), _p(self.u),
                                                                    _p(self.rho))
        self.g[...] = self.f
        self.v[...] = self.u
        self.rhob[...] = self.rho

    def step(self, params, n=1, collect=False, accumulate=False):
        """n steps; with `collect` the last step's momentum exchange is kept (added to the previous
        collection when `accumulate`, as the sub-steps of a refined level add up)."""
        suf = _suffix(self.dtype)
        for s in range(n):
            if self.desc is None:
                getattr(lib(), f"ora_q19_step_{suf}")(self.nocts, _p(self.onbr), C.addressof(params), _p(self.f),
                                                      _p(self.g), _p(self.u), _p(self.v), _p(self.rho), _p(self.rhob))
            else:
                mom = self.mom if (collect and s == n - 1) else None
                if mom is not None and not accumulate:
                    mom[...] = 0.0
                getattr(lib(), f"ora_q19_step_walls_{suf}")(C.addressof(self.desc), C.addressof(params), _p(self.f),
                                                            _p(self.g), _p(self.u), _p(self.v), _p(self.rho),
                                                            _p(self.rhob), _p(mom))
                if mom is not None:
                    self.per_tri = np.zeros((max(self.desc.ntri, 1), 3))
                    lib().ora_q19_forces(C.addressof(self.desc), _p(self.mom), _p(self.per_tri), _p(self.forces))
            self.f, self.g = self.g, self.f
            self.u, self.v = self.v, self.u
            self.rho, self.rhob = self.rhob, self.rho
        return self

    def totals(self):
        r = self.rho.astype(np.float64)
        u = self.u.astype(np.float64)
        if self.kind is not None:
            fl = (self.kind.reshape(self.nocts, 8) == 1)
            r = r * fl
            u = u * fl[:, None, :]
        return np.array([r.sum(), (r * u[:, 0]).sum(), (r * u[:, 1]).sum(), (r * u[:, 2]).sum(),
                         0.5 * (r * (u ** 2).sum(1)).sum()])


class OracleQ19Octree:
    """Several octree levels coupled by the oracle's transfers, stepped as the reference's
    step_recursive! (coupling.jl:240-254); `descs` are the levels' descriptors (kept alive by the
    caller), `params` one oal_q19_params per level."""

    def __init__(self, descs, onbrs, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self.descs = descs
        self.levels = [OracleQ19Level(o, dtype, desc=d) for o, d in zip(onbrs, descs)]
        self.L = len(self.levels)
        self.ghosts = [np.ctypeslib.as_array((C.c_int32 * d.nghost).from_address(d.ghost_slot)).copy() - 1
                       if d.nghost else np.zeros(0, np.int64) for d in descs]
        self.forces = np.zeros(3)
        self.per_tri = None

    def _fill(self, l, weight, params):
        F, Cl = self.levels[l - 1], self.levels[l - 2]
        getattr(lib(), f"ora_q19_fill_{_suffix(self.dtype)}")(
            C.addressof(self.descs[l - 1]), _p(Cl.kind), _p(Cl.f), _p(Cl.g), float(weight), float(params[l - 2].nu),
            float(params[l - 1].nu), _p(F.f), _p(F.u), _p(F.rho))

    def _restrict(self, l, params):
        Cl, F = self.levels[l - 1], self.levels[l]
        getattr(lib(), f"ora_q19_restrict_{_suffix(self.dtype)}")(
            C.addressof(self.descs[l - 1]), _p(F.f), float(params[l - 1].nu), float(params[l].nu), _p(Cl.f), _p(Cl.u),
            _p(Cl.rho))

    def _copy_ghosts(self, l):
        if l == self.L or not len(self.ghosts[l - 1]):
            return
        S = self.levels[l - 1]
        o, k = self.ghosts[l - 1] // 8, self.ghosts[l - 1] % 8
        S.f[o, :, k] = S.g[o, :, k]
        S.u[o, :, k] = S.v[o, :, k]
        S.rho[o, k] = S.rhob[o, k]

    @staticmethod
    def _mirror(S):
        S.g[...] = S.f
        S.v[...] = S.u
        S.rhob[...] = S.rho

    def initialise(self, params, fields):
        """fields[l] = (rho, u, du) of level l + 1; then couple_initial! (coupling.jl:257-268)."""
        for S, p, (rho, u, du) in zip(self.levels, params, fields):
            S.initialise(p, rho, u, du)
        for l in range(self.L - 1, 0, -1):
            self._restrict(l, params)
            self._mirror(self.levels[l - 1])
        for l in range(2, self.L + 1):
            self._fill(l, 1.0, params)
            self._mirror(self.levels[l - 1])

    def _step_recursive(self, l, params, collect):
        self.levels[l - 1].step(params[l - 1], 1, collect=collect, accumulate=True)
        self._copy_ghosts(l)
        if l < self.L:
            self._step_recursive(l + 1, params, collect)
            self._restrict(l, params)
            self._fill(l + 1, 0.5, params)
            self._step_recursive(l + 1, params, collect)
            self._restrict(l, params)
            self._fill(l + 1, 1.0, params)

    def advance(self, params, n=1, collect=False):
        for s in range(n):
            last = collect and s == n - 1
            if last:
                for S in self.levels:
                    S.mom[...] = 0.0
            self._step_recursive(1, params, last)
            if last:
                ntri = max(max(d.ntri for d in self.descs), 1)
                self.per_tri = np.zeros((ntri, 3))
                for S, d in zip(self.levels, self.descs):
                    pt = np.zeros((max(d.ntri, 1), 3))
                    tot = np.zeros(3)
                    if d.nlinks:
                        lib().ora_q19_forces(C.addressof(d), _p(S.mom), _p(pt), _p(tot))
                    self.per_tri[:pt.shape[0]] += pt
                self.forces = self.per_tri.sum(0)

    def totals(self):
        out = np.zeros(5)
        for l, S in enumerate(self.levels, start=1):
            out += 8.0 ** (self.L - l) * S.totals()
        return out


# ---- D3Q39 entropic KBC (oal_oracle_q39.cpp) ------------------------------------------------------

def q39_tables():
    cx, cy, cz, opp = (np.zeros(39, np.int32) for _ in range(4))
    w = np.zeros(39, np.float32)
    lib().ora_q39_tables(_p(cx), _p(cy), _p(cz), _p(w), _p(opp))
    return dict(cx=cx, cy=cy, cz=cz, w=w, opp=opp)


def q39_exp(x):
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    lib().ora_q39_exp(x.size, _p(x), _p(y))
    return y


def q39_log(x):
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    lib().ora_q39_log(x.size, _p(x), _p(y))
    return y


def q39_equilibrium(rho, u):
    """13-moment equilibrium from the polynomial start: rho (n,), u (n,3) -> feq (n,39), lambda (n,13)."""
    rho = np.ascontiguousarray(rho, np.float32)
    u = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
    n = rho.size
    feq = np.zeros((n, 39), np.float32)
    lam = np.zeros((n, 13), np.float32)
    lib().ora_q39_equilibrium(n, _p(rho), _p(u), _p(feq), _p(lam))
    return feq, lam


def q39_inlet_equilibrium(u_inlet):
    out = np.zeros(39, np.float32)
    lib().ora_q39_inlet_equilibrium(float(u_inlet), _p(out))
    return out


def q39_collide(params, f, g, lam):
    """Collision of independent cells: f (n,39), g (n,9) with g[3a+b] = d u_a / d x_b, lam (n,13)
    (NaN row = no warm start) -> (f_out, rho, u, lam_out)."""
    f = np.ascontiguousarray(f, np.float32)
    n = f.shape[0]
    g = np.ascontiguousarray(g, np.float32)
    lam = np.array(lam, np.float32, copy=True, order="C")
    fo = np.zeros_like(f)
    rho = np.zeros(n, np.float32)
    u = np.zeros((n, 3), np.float32)
    lib().ora_q39_collide_cells(n, C.addressof(params), _p(f), _p(g), _p(lam), _p(fo), _p(rho), _p(u))
    return fo, rho, u, lam


class OracleQ39Level:
    """D3Q39 entropic level in the reference layout, stepped by the CPU restatement (float32):
    f (39, nb, 512), rho (nb, 512), vel (3, nb, 512), lam (13, nb, 512) with NaN = no warm start;
    nbr (27, nb) 1-based. Without `coords` every neighbour must be present (periodic box); with
    `coords` (nb, 3, 1-based block coordinates) and `shape` (cells) missing neighbours are domain
    faces, and `obstacle` (nb, 512) marks solid cells."""

    def __init__(self, nbr, coords=None, shape=None, obstacle=None, sponge=None, wall_dist=None):
        self.nbr = np.ascontiguousarray(nbr, np.int32)
        self.nb = self.nbr.shape[1]
        self.coords = None if coords is None else np.ascontiguousarray(coords, np.int32)
        self.shape = shape
        self.obstacle = None if obstacle is None else np.ascontiguousarray(obstacle, np.uint8)
        self.sponge = None if sponge is None else np.ascontiguousarray(sponge, np.float32)
        self.wall_dist = None if wall_dist is None else np.ascontiguousarray(wall_dist, np.float32)
        nb = self.nb
        self.f = np.zeros((39, nb, 512), np.float32)
        self.g = np.zeros_like(self.f)
        self.rho = np.ones((nb, 512), np.float32)
        self.vel = np.zeros((3, nb, 512), np.float32)
        self.vel_new = np.zeros_like(self.vel)
        self.lam = np.full((13, nb, 512), np.nan, np.float32)

    def init_equilibrium(self, rho, vel):
        rho = np.asarray(rho, np.float32).reshape(self.nb * 512)
        vel = np.asarray(vel, np.float32).reshape(3, self.nb * 512)
        feq, _ = q39_equilibrium(rho, vel.T)
        self.f[...] = feq.T.reshape(39, self.nb, 512)
        self.rho[...] = rho.reshape(self.nb, 512)
        self.vel[...] = vel.reshape(3, self.nb, 512)
        self.lam[...] = np.nan
        return self

    def step(self, params, n=1):
        for _ in range(n):
            if self.coords is None:
                lib().ora_q39_step(self.nb, _p(self.nbr), C.addressof(params), _p(self.f), _p(self.g), _p(self.vel),
                                   _p(self.vel_new), _p(self.rho), _p(self.lam))
            else:
                nx, ny, nz = self.shape
                lib().ora_q39_step_ex(self.nb, _p(self.nbr), _p(self.coords), nx, ny, nz,
                                      None if self.obstacle is None else _p(self.obstacle), _p(self.sponge),
                                      _p(self.wall_dist), C.addressof(params),
                                      _p(self.f), _p(self.g), _p(self.vel), _p(self.vel_new), _p(self.rho),
                                      _p(self.lam))
            self.f, self.g = self.g, self.f
            self.vel, self.vel_new = self.vel_new, self.vel
        return self

    def mass_momentum(self):
        t = q39_tables()
        f = self.f.astype(np.float64)
        c = np.stack([t["cx"], t["cy"], t["cz"]]).astype(np.float64)
        return np.array([f.sum(), *(np.tensordot(c, f, axes=(1, 0)).sum(axis=(1, 2)))])
