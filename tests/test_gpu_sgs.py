"""Variable eddy viscosity of the CUDA D3Q27 step against the oracle (kernel_cumulant.jl:546-588):
mode 1, nu_sgs from the previous step's post-collision Pi_neq (refresh_pi_neq!, fused into the
general kernel's store); mode 2, the Germano-Lilly dynamic coefficient (kernel_dynamic_sgs.jl).
Tolerances as the plain step's: FP64 1e-11, FP32 2e-5, FP16 deviation storage 2e-3 of max |f|
against the FP64 oracle. The Pi_neq diagnostic (oal_level_pi_neq) against the oracle's; graph
replay against single steps; the refusals of the paths that hold no Pi_neq field.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200.cases import sphere_channel_case, taylor_green_case
from openaerolab_alpha_01_b200.solver import Batch, Geometry, Level


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))) / np.max(np.abs(b)))


def with_sgs(params, mode, floor=0.0, c_pi=0.2):
    p = capi.StepParams.from_buffer_copy(params)
    p.variable_nu_sgs = mode
    p.nu_sgs_floor = floor
    p.c_pi = c_pi
    return p


def run_pair(oracle, case, p, storage, dtype, steps, layout="block"):
    g = Geometry(case.dom)
    L = Level(g, storage=storage, layout=layout)
    L.init_equilibrium(case.rho, case.vel)
    d = case.dom
    O = oracle.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, sponge=d.sponge,
                           wall_dist=d.wall_dist, dtype=dtype)
    O.init_equilibrium(case.rho, case.vel)
    for i in range(steps):
        p.time_step_seed = i
        L.perform_timestep(p)
        O.step(p)
    f, rho, vel = L.state()
    out = dict(f=f, rho=rho, vel=vel, force=L.forces() if p.collect_forces else None, pi=L.pi_neq())
    L.close(); g.close()
    return out, O


@pytest.fixture(scope="module")
def tgv():
    return taylor_green_case(16, u0=0.08, re=200.0, c_wale=0.2)


@pytest.fixture(scope="module")
def channel():
    return sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("storage,dtype,tol,layout", [("f64", np.float64, 1e-11, "block"),
                                                      ("f32", np.float32, 2e-5, "block"),
                                                      ("f32", np.float32, 2e-5, "dense"),
                                                      ("f16", np.float64, 2e-3, "block")])
def test_taylor_green(oal, oracle_lib, tgv, mode, storage, dtype, tol, layout):
    p = with_sgs(tgv.params, mode)
    g, O = run_pair(oracle_lib, tgv, p, storage, dtype, 16, layout)
    assert rel(g["f"], O.f) < tol
    assert rel(g["vel"], O.vel) < tol * 50
    if mode == 1 and storage != "f16":
        # the refreshed field is the stored state's Pi_neq: the diagnostic reads it back
        assert np.max(np.abs(g["pi"] - O.pi_neq)) < 4e-7 + tol * np.max(np.abs(O.pi_neq))


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("storage,dtype,tol,ftol", [("f64", np.float64, 1e-11, 1e-10),
                                                    ("f32", np.float32, 2e-5, 1e-4)])
def test_sphere_channel_halfway(oal, oracle_lib, channel, mode, storage, dtype, tol, ftol):
    p = with_sgs(channel.params, mode, floor=0.002)
    g, O = run_pair(oracle_lib, channel, p, storage, dtype, 12)
    assert rel(g["f"], O.f) < tol
    assert abs(g["force"][0] - O.force[0]) <= ftol * abs(O.force[0])
    assert np.all(g["pi"][:, channel.dom.obstacle == 1] == 0)


@pytest.mark.parametrize("storage,dtype,tol", [("f64", np.float64, 1e-11), ("f32", np.float32, 2e-5)])
def test_grad_wall_and_compressible(oal, oracle_lib, channel, storage, dtype, tol):
    p = with_sgs(channel.params, 1)
    p.solid_bc = capi.OAL_SOLID_GRAD
    p.collect_forces = 0
    p.compressible_corr = 1
    g, O = run_pair(oracle_lib, channel, p, storage, dtype, 10)
    assert rel(g["f"], O.f) < tol
    assert np.max(np.abs(g["pi"] - O.pi_neq)) < 4e-7 + tol * np.max(np.abs(O.pi_neq))


def test_bouzidi_refreshes_pi_after_the_correction(oal, oracle_lib, channel):
    from openaerolab_alpha_01_b200.bouzidi import sphere_qmap
    d = channel.dom
    cells, q = sphere_qmap(d, (10.0, 8.0, 8.0), 3.0)
    bz = dict(cells=cells, q=q)
    p = with_sgs(channel.params, 1)
    p.solid_bc = capi.OAL_SOLID_BOUZIDI
    p.collect_forces = 0
    g = Geometry(d)
    L = Level(g, storage="f64")
    L.init_equilibrium(channel.rho, channel.vel)
    L.set_bouzidi(cells, q)
    O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, dtype=np.float64)
    O.init_equilibrium(channel.rho, channel.vel)
    for _ in range(10):
        L.perform_timestep(p)
        O.step_bouzidi(p, bz)
    f = L.state()[0]
    pi = L.pi_neq()
    L.close(); g.close()
    assert rel(f, O.f) < 1e-11
    assert np.max(np.abs(pi - O.pi_neq)) < 4e-7


def test_pi_neq_diagnostic_of_the_plain_step(oal, oracle_lib, channel):
    """oal_level_pi_neq on a level stepped without variable nu_sgs (compute_pi_neq_for_level!)."""
    g, O = run_pair(oracle_lib, channel, capi.StepParams.from_buffer_copy(channel.params), "f64", np.float64, 8)
    ref = O.state_pi_neq()
    assert np.max(np.abs(g["pi"] - ref)) < 4e-7
    assert np.max(np.abs(ref)) > 1e-5


@pytest.mark.parametrize("mode", [1, 2])
def test_graph_advance_equals_single_steps(oal, channel, mode):
    p = with_sgs(channel.params, mode)
    g = Geometry(channel.dom)
    A = Level(g, storage="f32")
    B = Level(g, storage="f32")
    A.init_equilibrium(channel.rho, channel.vel)
    B.init_equilibrium(channel.rho, channel.vel)
    for _ in range(7):
        A.perform_timestep(p)
    B.execute_timestep_batch(p, 7)
    assert np.array_equal(A.state()[0], B.state()[0])
    assert np.array_equal(A.pi_neq(), B.pi_neq())
    assert np.array_equal(A.forces(), B.forces())
    A.close(); B.close(); g.close()


def test_refusals(oal, channel):
    g = Geometry(channel.dom)
    L = Level(g)
    L.init_equilibrium(channel.rho, channel.vel)
    p = with_sgs(channel.params, 3)
    with pytest.raises(capi.OALError) as e:
        L.perform_timestep(p)
    assert e.value.status == capi.OAL_E_INVALID_ARG
    L.close()
    B = Batch(storage="f32", max_real_blocks=64, max_ghost_blocks=64, max_mask_blocks=16, max_members=2)
    for mode in (1, 2):
        with pytest.raises(capi.OALError) as e:
            B.add(g, with_sgs(channel.params, mode), channel.rho, channel.vel)
        assert e.value.status == capi.OAL_E_UNSUPPORTED
    B.close()
    nb = channel.dom.n_blocks
    fl = capi.LevelFields(None, None, None, None, None, None, capi.OAL_STORE_F32, 0, 512, 512 * nb, 512 * nb, None)
    with pytest.raises(capi.OALError) as e:
        capi.check(capi.lib().oal_stream_collide(g.handle, C.byref(fl), C.byref(with_sgs(channel.params, 2)), None))
    assert e.value.status == capi.OAL_E_UNSUPPORTED
    g.close()
