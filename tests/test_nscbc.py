"""Characteristic (NSCBC) outlet (apply_nscbc_outlet_kernel! / apply_nscbc_outlet!,
src/collision/kernel_nscbc_outlet.jl:80-393), athermal.

CPU: the oracle's restatement against closed forms: a uniform stream at the target pressure is
left as it is; a uniform density excess relaxes by the LODI rate d rho = K (1 - M^2)(p - p_t) /
(2 c^2); corner cells keep the interior's tangential velocity; only the x = 8 plane of the +x
blocks changes (every block's x = 8 plane with all_blocks). GPU: the level's outlet after each
step against the oracle's step + outlet (FP64 1e-11, FP32 2e-5), with the Pi_neq re-refresh, and
graph replay equal to single steps.
"""
import math

import numpy as np
import pytest

from openaerolab_alpha_01_b200.cases import sphere_channel_case


def box(oracle, nbx=3, nby=2, nbz=2, rho0=1.0, u=(0.05, 0.0, 0.0), dtype=np.float64):
    coords, nbr = oracle.build_box(nbx, nby, nbz, 0)
    nb = coords.shape[0]
    rho = np.full((nb, 512), rho0)
    vel = np.zeros((3, nb, 512))
    for c in range(3):
        vel[c] = u[c]
    O = oracle.OracleLevel(coords, nbr, (8 * nbx, 8 * nby, 8 * nbz), dtype=dtype)
    O.init_equilibrium(rho, vel)
    return O


def face_mask(O, all_blocks=False):
    lx = np.arange(512) & 7
    bx = O.coords[:, 0]
    sel = (bx == bx.max()) if not all_blocks else np.ones_like(bx, bool)
    return sel[:, None] & (lx[None, :] == 7)


def test_uniform_stream_at_target_pressure_is_kept(oracle_lib):
    O = box(oracle_lib)
    f0, r0, v0 = O.f.copy(), O.rho.copy(), O.vel.copy()
    O.nscbc(p_target=float(np.float32(1.0 / 3.0)))
    assert np.max(np.abs(O.rho - r0)) < 1e-7 and np.max(np.abs(O.vel - v0)) < 1e-9
    assert np.max(np.abs(O.f - f0)) < 1e-8


def test_density_excess_relaxes_at_the_lodi_rate(oracle_lib):
    rho0, u = 1.01, 0.05
    O = box(oracle_lib, rho0=rho0, u=(u, 0.0, 0.0))
    nx = O.shape[0]
    r0 = O.rho.copy()
    O.nscbc(p_target=1.0 / 3.0, sigma_relax=0.27)
    c = math.sqrt(1.0 / 3.0)
    K = np.float32(0.27) * np.float32(math.sqrt(np.float32(2.0 / 3.0))) / np.float32(nx)
    M = u / c
    L1 = float(K) * (1 - M * M) * (rho0 / 3.0 - float(np.float32(1.0 / 3.0)))
    # no gradients: L2 = L3 = L4 = 0, L5 = 0, d1 = L1 / (2 c^2), d3 = -L1 / (2 rho c)
    m = face_mask(O)
    expect = rho0 - L1 / (2 * c * c)
    assert np.allclose(O.rho[m], expect, rtol=0, atol=1e-12)
    assert np.array_equal(O.rho[~m], r0[~m])
    assert np.allclose(O.vel[0][m], u + L1 / (2 * rho0 * c), rtol=0, atol=1e-12)


def test_corners_keep_the_interior_tangential_velocity(oracle_lib):
    O = box(oracle_lib, u=(0.05, 0.0, 0.0))
    lx, ly, lz = np.arange(512) & 7, (np.arange(512) >> 3) & 7, np.arange(512) >> 6
    gy = (O.coords[:, 1:2] - 1) * 8 + ly[None] + 1
    # a tangential shear in x: the interior plane x = 7 carries v = 0.01, the face v = 0.02
    O.vel[1] = np.where(lx[None] == 6, 0.01, 0.0) + np.where(lx[None] == 7, 0.02, 0.0)
    O.nscbc(p_target=1.0 / 3.0)
    m = face_mask(O)
    corner = m & ((gy == 1) | (gy == O.shape[1]))
    inner = m & ~corner & (((O.coords[:, 2:3] - 1) * 8 + lz[None] + 1) > 1) & \
        (((O.coords[:, 2:3] - 1) * 8 + lz[None] + 1) < O.shape[2])
    assert np.all(O.vel[1][corner] == 0.01)
    c = math.sqrt(1.0 / 3.0)
    L3 = 0.05 * (0.02 - 0.01)
    assert np.allclose(O.vel[1][inner], 0.02 - min(L3, 0.1 * c), atol=1e-15)


def test_all_blocks_touches_every_block_plane(oracle_lib):
    O = box(oracle_lib, rho0=1.01)
    r0 = O.rho.copy()
    O.nscbc(all_blocks=True, p_target=1.0 / 3.0)
    m = face_mask(O, all_blocks=True)
    assert np.all(O.rho[m] != r0[m]) and np.array_equal(O.rho[~m], r0[~m])


def _level_vs_oracle(oal, oracle, case, storage, dtype, steps, all_blocks, params=None):
    from openaerolab_alpha_01_b200.solver import Geometry, Level
    d = case.dom
    g = Geometry(d)
    L = Level(g, storage=storage)
    L.init_equilibrium(case.rho, case.vel)
    L.set_nscbc(True, all_blocks=all_blocks, p_target=1.0 / 3.0, sigma_relax=0.27, neq_blend=0.5)
    O = oracle.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, sponge=d.sponge,
                           wall_dist=d.wall_dist, dtype=dtype)
    O.init_equilibrium(case.rho, case.vel)
    p = params or case.params
    for _ in range(steps):
        L.perform_timestep(p)
        O.step(p)
        O.nscbc(all_blocks=all_blocks, p_target=1.0 / 3.0)
        if p.variable_nu_sgs == 1:
            O.pi_neq[...] = O.state_pi_neq(p.compressible_corr)
    f, rho, vel = L.state()
    pi = L.pi_neq()
    L.close(); g.close()
    return f, rho, vel, pi, O


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))) / np.max(np.abs(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("all_blocks", [False, True])
@pytest.mark.parametrize("storage,dtype,tol", [("f64", np.float64, 1e-11), ("f32", np.float32, 2e-5)])
def test_gpu_outlet_matches_oracle(oal, oracle_lib, storage, dtype, tol, all_blocks):
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    f, rho, vel, _, O = _level_vs_oracle(oal, oracle_lib, case, storage, dtype, 10, all_blocks)
    assert rel(f, O.f) < tol
    assert rel(rho, O.rho) < tol and rel(vel, O.vel) < tol * 50


@pytest.mark.gpu
def test_gpu_outlet_with_pi_neq_sgs(oal, oracle_lib):
    from openaerolab_alpha_01_b200 import _capi as capi
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    p = capi.StepParams.from_buffer_copy(case.params)
    p.variable_nu_sgs = 1
    p.nu_sgs_floor = 0.0
    f, rho, vel, pi, O = _level_vs_oracle(oal, oracle_lib, case, "f64", np.float64, 8, False, p)
    assert rel(f, O.f) < 1e-11
    assert np.max(np.abs(pi - O.pi_neq)) < 4e-7


@pytest.mark.gpu
@pytest.mark.parametrize("storage,dtype,tol", [("f64", np.float64, 1e-11), ("f32", np.float32, 2e-5)])
def test_gpu_outlet_after_the_svv_filter(oal, oracle_lib, storage, dtype, tol):
    """The filter, then the outlet (timestep.jl:1576-1611 before :1617-1664): the outlet rebuilds
    its face plane from the filtered state."""
    from openaerolab_alpha_01_b200 import _capi as capi
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    p = capi.StepParams.from_buffer_copy(case.params)
    p.svv_x_epsilon = 0.003
    p.svv_yz_epsilon = 0.005
    f, rho, vel, _, O = _level_vs_oracle(oal, oracle_lib, case, storage, dtype, 8, False, p)
    assert rel(f, O.f) < tol
    assert rel(rho, O.rho) < tol and rel(vel, O.vel) < tol * 50


@pytest.mark.gpu
def test_gpu_outlet_graph_replay(oal):
    from openaerolab_alpha_01_b200.solver import Geometry, Level
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    g = Geometry(case.dom)
    A, B = Level(g, storage="f16"), Level(g, storage="f16")
    for X in (A, B):
        X.init_equilibrium(case.rho, case.vel)
        X.set_nscbc(True, p_target=1.0 / 3.0)
    for _ in range(6):
        A.perform_timestep(case.params)
    B.execute_timestep_batch(case.params, 6)
    assert np.array_equal(A.state()[0], B.state()[0])
    B.set_nscbc(False)
    A.close(); B.close(); g.close()
