"""CUDA D3Q27 cumulant step against the CPU oracle (a restatement of kernel_cumulant.jl) on the same
seeded inputs. Tolerances (relative to max |f|, per comparison):

* FP64 storage vs FP64 oracle ............ 1e-11 (only fused multiply-add rounding differs)
* FP32 storage vs FP32 oracle ............ 2e-5 over 20-30 steps
* FP16 / BF16 deviation storage vs FP64 .. 2e-3 / 2e-2 of max |f|, drag within 0.5 % / 5 %
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200.cases import sphere_channel_case, taylor_green_case
from openaerolab_alpha_01_b200.solver import Geometry, Level


def run_gpu(case, storage, steps, params=None, layout="block"):
    g = Geometry(case.dom)
    L = Level(g, storage=storage, layout=layout)
    L.init_equilibrium(case.rho, case.vel)
    p = params or case.params
    for i in range(steps):
        p.time_step_seed = i
        L.perform_timestep(p)
    f, rho, vel = L.state()
    force = L.forces()
    mm = L.mass_momentum()
    L.close(); g.close()
    return f, rho, vel, force, mm


def run_oracle(oracle, case, steps, dtype=np.float64, params=None):
    d = case.dom
    O = oracle.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, sponge=d.sponge,
                           wall_dist=d.wall_dist, dtype=dtype)
    O.init_equilibrium(case.rho, case.vel)
    p = params or case.params
    for i in range(steps):
        p.time_step_seed = i
        O.step(p)
    return O


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def tgv():
    return taylor_green_case(16, u0=0.05, re=100.0, c_wale=0.2)


@pytest.mark.parametrize("layout", ["block", "dense"])
@pytest.mark.parametrize("storage,dtype,tol", [("f64", np.float64, 1e-11), ("f32", np.float32, 2e-5),
                                               ("f16", np.float64, 2e-3), ("bf16", np.float64, 2e-2)])
def test_taylor_green_periodic(oal, oracle_lib, tgv, storage, dtype, tol, layout):
    # a periodic box; the dense layout (FP32/FP16/BF16) copies the periodic ghost frame
    steps = 20
    f, rho, vel, _, mm = run_gpu(tgv, storage, steps, layout=layout)
    O = run_oracle(oracle_lib, tgv, steps, dtype)
    assert rel(f, O.f) < tol
    assert rel(vel, O.vel) < tol * 50
    assert rel(rho, O.rho) < tol
    om = O.mass_momentum()
    assert abs(mm[0] - om[0]) / om[0] < max(tol, 1e-12)


@pytest.fixture(scope="module")
def channel():
    return sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)


@pytest.mark.parametrize("storage,dtype,tol,ftol,sym", [("f64", np.float64, 1e-11, 1e-10, 1e-9),
                                                        ("f32", np.float32, 2e-5, 1e-4, 1e-4),
                                                        ("f16", np.float64, 2e-3, 5e-3, 1e-3),
                                                        ("bf16", np.float64, 2e-2, 5e-2, 1e-2)])
@pytest.mark.parametrize("layout", ["block", "dense"])
def test_sphere_channel_halfway_drag(oal, oracle_lib, channel, storage, dtype, tol, ftol, sym, layout):
    steps = 30
    f, rho, vel, force, _ = run_gpu(channel, storage, steps, layout=layout)
    O = run_oracle(oracle_lib, channel, steps, dtype)
    assert rel(f, O.f) < tol
    assert abs(force[0] - O.force[0]) / abs(O.force[0]) < ftol
    # the sphere is centred in y and z: the side forces vanish up to storage rounding
    assert abs(force[1]) < sym * abs(force[0]) + 1e-12
    assert abs(force[2]) < sym * abs(force[0]) + 1e-12


VARIANTS = {
    "fullway": dict(solid_bc=capi.OAL_SOLID_FULLWAY, collect_forces=0),
    "zwall_slip": dict(zwall_bc=1),
    "zwall_noslip": dict(zwall_bc=2),
    "ymin_wall": dict(ymin_wall_bc=1),
    "transverse_freestream": dict(transverse_freestream=1, transverse_freestream_blend=0.5),
    "inlet_noise": dict(inlet_turbulence=0.05),
    "positivity_limiter": dict(limiter_type=capi.OAL_LIMITER_POSITIVITY),
    "no_limiter_fixed_omega4": dict(limiter_type=capi.OAL_LIMITER_NONE, adaptive_omega4=0, omega4=0.8),
    "relaxation_rates": dict(omega_bulk=0.7, omega3=0.9, nu_sgs_background=1e-3),
    "compressible": dict(compressible_corr=1),
    "no_wale": dict(c_wale=0.0),
    "grad_wall": dict(solid_bc=capi.OAL_SOLID_GRAD, collect_forces=0),
    "grad_wall_half_stress": dict(solid_bc=capi.OAL_SOLID_GRAD, collect_forces=0, grad_pineq_scale=0.5),
}


# Every branch on both population layouts: block-major with ghost blocks, and the dense padded
# grid with its ghost frame (FP32).
@pytest.mark.parametrize("storage,dtype,tol,vtol,ftol,layout", [("f64", np.float64, 1e-11, 1e-9, 1e-10, "block"),
                                                                ("f32", np.float32, 2e-5, 5e-4, 1e-4, "block"),
                                                                ("f32", np.float32, 2e-5, 5e-4, 1e-4, "dense")])
@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_boundary_and_option_branches(oal, oracle_lib, channel, name, storage, dtype, tol, vtol, ftol, layout):
    p = capi.default_params(**{f: getattr(channel.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    for k, v in VARIANTS[name].items():
        setattr(p, k, v)
    steps = 12
    f, rho, vel, force, _ = run_gpu(channel, storage, steps, params=p, layout=layout)
    O = run_oracle(oracle_lib, channel, steps, dtype, params=p)
    assert rel(f, O.f) < tol, name
    assert rel(vel, O.vel) < vtol, name
    if p.collect_forces:
        assert abs(force[0] - O.force[0]) <= ftol * abs(O.force[0]), name


@pytest.mark.parametrize("storage,dtype,tol,layout", [("f64", np.float64, 1e-10, "block"),
                                                      ("f32", np.float32, 2e-5, "block"),
                                                      ("f32", np.float32, 2e-5, "dense")])
def test_sponge_and_wall_model(oal, oracle_lib, storage, dtype, tol, layout):
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=200.0)
    d = case.dom
    gx, gy, gz = d.cell_positions()
    d.sponge = np.clip((gx - 24.0) / 8.0, 0.0, 1.0).astype(np.float32) * 0.5
    r = np.sqrt((gx - 0.5 - 10.0) ** 2 + (gy - 0.5 - 8.0) ** 2 + (gz - 0.5 - 8.0) ** 2) - 3.0
    d.wall_dist = np.where(d.obstacle != 0, 0.0, np.maximum(r, 0.0)).astype(np.float32)
    p = case.params
    p.sponge_blend_distributions = 1
    p.wall_model_active = 1
    p.wall_model_max_distance = 4.0
    steps = 12
    f, rho, vel, force, _ = run_gpu(case, storage, steps, params=p, layout=layout)
    O = run_oracle(oracle_lib, case, steps, dtype, params=p)
    assert rel(f, O.f) < tol
    assert rel(rho, O.rho) < tol


@pytest.mark.parametrize("layout", ["block", "dense"])
def test_graph_advance_equals_single_steps(oal, layout):
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    g = Geometry(case.dom)
    A = Level(g, storage="f32", layout=layout)
    B = Level(g, storage="f32", layout=layout)
    A.init_equilibrium(case.rho, case.vel)
    B.init_equilibrium(case.rho, case.vel)
    for _ in range(7):
        A.perform_timestep(case.params)
    B.execute_timestep_batch(case.params, 7)
    fa, ra, va = A.state()
    fb, rb, vb = B.state()
    assert np.array_equal(fa, fb) and np.array_equal(va, vb)
    assert np.array_equal(A.forces(), B.forces())
    B.execute_timestep_batch(case.params, 7)  # cached graph, other parity
    for _ in range(7):
        A.perform_timestep(case.params)
    assert np.array_equal(A.state()[0], B.state()[0])


def test_caller_owned_arrays_reference_layout(oal, oracle_lib):
    """oal_stream_collide on torch-owned arrays in the reference's (8,8,8,nb,27) layout."""
    import torch
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    oracle = oracle_lib
    g = Geometry(case.dom)
    nb = case.dom.n_blocks
    f0 = oracle.init_feq(case.rho, case.vel)
    fa = torch.tensor(f0, dtype=torch.float32, device="cuda").contiguous()
    fb = torch.empty_like(fa)
    va = torch.tensor(case.vel, dtype=torch.float32, device="cuda").contiguous()
    vb = torch.empty_like(va)
    rho = torch.empty((nb, 512), dtype=torch.float32, device="cuda")
    force = torch.zeros(3, dtype=torch.float64, device="cuda")
    p = case.params
    steps = 10
    for i in range(steps):
        fl = capi.LevelFields(fa.data_ptr(), fb.data_ptr(), None, rho.data_ptr(), vb.data_ptr(), va.data_ptr(),
                              capi.OAL_STORE_F32, 0, 512, 512 * nb, 512 * nb, force.data_ptr())
        capi.check(capi.lib().oal_stream_collide(g.handle, C.byref(fl), C.byref(p), None))
        fa, fb = fb, fa
        va, vb = vb, va
    torch.cuda.synchronize()
    O = run_oracle(oracle, case, steps, np.float32)
    assert rel(fa.cpu().numpy(), O.f) < 2e-5
    assert abs(force[0].item() - O.force[0]) / abs(O.force[0]) < 1e-4


@pytest.mark.parametrize("solid_bc", [capi.OAL_SOLID_FULLWAY, capi.OAL_SOLID_HALFWAY])
def test_store_post_collision_on_caller_arrays(oal, oracle_lib, solid_bc):
    """kernel_cumulant.jl:889-908: with store_post_collision the post-collision populations are
    also written to f_post_collision (every cell, solid ones included); the Bouzidi correction
    reads them from there."""
    import torch
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    g = Geometry(case.dom)
    nb = case.dom.n_blocks
    p = capi.default_params(**{f: getattr(case.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    p.solid_bc = solid_bc
    p.store_post_collision = 1
    f0 = oracle_lib.init_feq(case.rho, case.vel)
    fa = torch.tensor(f0, dtype=torch.float32, device="cuda").contiguous()
    fb = torch.empty_like(fa)
    post = torch.full_like(fa, float("nan"))
    va = torch.tensor(case.vel, dtype=torch.float32, device="cuda").contiguous()
    vb = torch.empty_like(va)
    rho = torch.empty((nb, 512), dtype=torch.float32, device="cuda")
    force = torch.zeros(3, dtype=torch.float64, device="cuda")
    steps = 6
    for i in range(steps):
        fl = capi.LevelFields(fa.data_ptr(), fb.data_ptr(), post.data_ptr(), rho.data_ptr(), vb.data_ptr(),
                              va.data_ptr(), capi.OAL_STORE_F32, 0, 512, 512 * nb, 512 * nb, force.data_ptr())
        capi.check(capi.lib().oal_stream_collide(g.handle, C.byref(fl), C.byref(p), None))
        fa, fb = fb, fa
        va, vb = vb, va
    torch.cuda.synchronize()
    g.close()
    got_post, got_f = post.cpu().numpy(), fa.cpu().numpy()
    assert not np.isnan(got_post).any()
    assert np.array_equal(got_post, got_f)
    O = run_oracle(oracle_lib, case, steps, np.float32, params=p)
    assert rel(got_post, O.f) < 2e-5


def test_caller_owned_arrays_with_bouzidi_walls(oal, oracle_lib):
    """oal_stream_collide with OAL_SOLID_BOUZIDI, then oal_bouzidi_apply on the caller's arrays
    (the reference's separate apply_bouzidi_correction! call), against the oracle's step +
    correction."""
    import torch
    from openaerolab_alpha_01_b200.bouzidi import sphere_qmap
    from openaerolab_alpha_01_b200.solver import BouzidiCells
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    d = case.dom
    cells, q = sphere_qmap(d, (10.0, 8.0, 8.0), 3.0)
    p = capi.default_params(**{f: getattr(case.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    p.solid_bc = capi.OAL_SOLID_BOUZIDI
    p.collect_forces = 0
    g = Geometry(d)
    bz = BouzidiCells(g, cells, q, storage="f32", ff_fallback=1)
    nb = d.n_blocks
    fa = torch.tensor(oracle_lib.init_feq(case.rho, case.vel), dtype=torch.float32, device="cuda").contiguous()
    fb = torch.empty_like(fa)
    va = torch.tensor(case.vel, dtype=torch.float32, device="cuda").contiguous()
    vb = torch.empty_like(va)
    rho = torch.empty((nb, 512), dtype=torch.float32, device="cuda")
    steps = 8
    for _ in range(steps):
        fl = capi.LevelFields(fa.data_ptr(), fb.data_ptr(), None, rho.data_ptr(), vb.data_ptr(), va.data_ptr(),
                              capi.OAL_STORE_F32, 0, 512, 512 * nb, 512 * nb, None)
        capi.check(capi.lib().oal_stream_collide(g.handle, C.byref(fl), C.byref(p), None))
        bz.apply(fl)
        fa, fb = fb, fa
        va, vb = vb, va
    torch.cuda.synchronize()
    O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, dtype=np.float32)
    O.init_equilibrium(case.rho, case.vel)
    for _ in range(steps):
        O.step_bouzidi(p, dict(cells=cells, q=q, ff_fallback=1))
    assert rel(fa.cpu().numpy(), O.f) < 2e-5
    bz.close()
    g.close()


def test_rejects_bad_params(oal):
    case = taylor_green_case(16)
    g = Geometry(case.dom)
    L = Level(g)
    L.init_equilibrium(case.rho, case.vel)
    p = capi.default_params(tau=0.5)
    with pytest.raises(capi.OALError) as e:
        L.perform_timestep(p)
    assert e.value.status == capi.OAL_E_INVALID_ARG
    p = capi.default_params(tau=0.6)
    p.abi_version = 99
    with pytest.raises(capi.OALError) as e:
        L.perform_timestep(p)
    assert e.value.status == capi.OAL_E_ABI_MISMATCH
    p = capi.default_params(tau=0.6, operator_id=capi.OAL_OP_ENTROPIC_D3Q39)
    with pytest.raises(capi.OALError) as e:
        L.perform_timestep(p)
    assert e.value.status == capi.OAL_E_UNSUPPORTED


BOUZIDI_OPTS = {"halfway_bb": {}, "wall_eq": dict(ff_fallback=1), "bounce_back": dict(ff_fallback=2),
                "limiter": dict(limiter_rel_cap=0.05, limiter_abs_cap=1e-4)}


# The linear Bouzidi wall (bc_scheme "bouzidi_linear") on the sphere's analytic q map, every
# fall-back and the wall-population limiter, on both layouts.
@pytest.mark.parametrize("storage,dtype,tol,layout", [("f64", np.float64, 1e-11, "block"),
                                                      ("f32", np.float32, 2e-5, "block"),
                                                      ("f32", np.float32, 2e-5, "dense"),
                                                      ("f16", np.float64, 2e-3, "block")])
@pytest.mark.parametrize("opt", sorted(BOUZIDI_OPTS))
def test_bouzidi_linear_wall(oal, oracle_lib, channel, opt, storage, dtype, tol, layout):
    from openaerolab_alpha_01_b200.bouzidi import sphere_qmap
    d = channel.dom
    cells, q = sphere_qmap(d, (10.0, 8.0, 8.0), 3.0)
    kw = BOUZIDI_OPTS[opt]
    p = capi.default_params(**{f: getattr(channel.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    p.solid_bc = capi.OAL_SOLID_BOUZIDI
    p.collect_forces = 0
    g = Geometry(d)
    L = Level(g, storage=storage, layout=layout)
    L.init_equilibrium(channel.rho, channel.vel)
    L.set_bouzidi(cells, q, **kw)
    O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, dtype=dtype)
    O.init_equilibrium(channel.rho, channel.vel)
    bz = dict(cells=cells, q=q, ff_fallback=kw.get("ff_fallback", 0), rel_cap=kw.get("limiter_rel_cap", 0.0),
              abs_cap=kw.get("limiter_abs_cap", 0.0))
    for i in range(12):
        p.time_step_seed = i
        L.perform_timestep(p)
        O.step_bouzidi(p, bz)
    f, rho, vel = L.state()
    L.close(); g.close()
    assert rel(f, O.f) < tol, opt
    assert rel(vel, O.vel) < tol * 50, opt


def test_bouzidi_graph_detach_and_refusals(oal, channel):
    from openaerolab_alpha_01_b200.bouzidi import sphere_qmap
    from openaerolab_alpha_01_b200.solver import Batch
    from openaerolab_alpha_01_b200._capi import OALError
    d = channel.dom
    cells, q = sphere_qmap(d, (10.0, 8.0, 8.0), 3.0)
    p = capi.default_params(**{f: getattr(channel.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    p.solid_bc = capi.OAL_SOLID_BOUZIDI
    p.collect_forces = 0
    g = Geometry(d)
    A, B, C_ = (Level(g, storage="f32") for _ in range(3))
    for X in (A, B, C_):
        X.init_equilibrium(channel.rho, channel.vel)
    A.set_bouzidi(cells, q)
    B.set_bouzidi(cells, q)
    for _ in range(6):
        A.perform_timestep(p)
    B.execute_timestep_batch(p, 6)  # the correction is captured with the step
    assert np.array_equal(A.state()[0], B.state()[0])
    # detached: OAL_SOLID_BOUZIDI without cells is the full-way step
    B.set_bouzidi(np.zeros((0, 4), np.int32), np.zeros((0, 27)))
    pf = capi.default_params(**{f: getattr(p, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    pf.solid_bc = capi.OAL_SOLID_FULLWAY
    C_.set_state(*B.state())
    B.execute_timestep_batch(p, 3)
    C_.execute_timestep_batch(pf, 3)
    assert np.array_equal(B.state()[0], C_.state()[0])
    bad = cells.copy()
    bad[0, 1] = 9
    with pytest.raises(OALError):
        A.set_bouzidi(bad, q)
    # the momentum exchange belongs to the full-way wall, not to the corrected links: refused
    pc = capi.default_params(**{f: getattr(p, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
    pc.collect_forces = 1
    with pytest.raises(OALError) as e:
        A.perform_timestep(pc)
    assert e.value.status == capi.OAL_E_UNSUPPORTED
    for X in (A, B, C_):
        X.close()
    g.close()
