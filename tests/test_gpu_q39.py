"""The D3Q39 entropic KBC level on the GPU against the oracle, bit for bit.

The kernel and the oracle evaluate the reference's step in the same IEEE binary32 operation order
(no contraction) with the same exp/log, so every population, density, velocity and cached
multiplier after each configuration's steps carries the oracle's bits. Configurations cover the
four alpha solvers, sigma damping, the HRR blend, the viscosity floors, the transonic branches
(Mach-pocket viscosity, macro realizability clamp, equilibrium velocity cap, realizability guards)
and the NaN reset. At a size the oracle would take minutes on, conservation and the shear-wave
viscosity are checked instead.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CS2 = 2.0 / 3.0


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.fixture(scope="module")
def env(oal, oracle_lib):
    from openaerolab_alpha_01_b200 import solver
    return oracle_lib, solver


def cell_xyz(dom):
    gx, gy, gz = dom.cell_positions()
    return gx - 1, gy - 1, gz - 1


def smooth_fields(dom, u0=0.05, seed=0, noise=0.01):
    X, Y, Z = cell_xyz(dom)
    nx, ny, nz = dom.shape
    rng = np.random.default_rng(seed)
    vel = np.zeros((3, dom.n_blocks, 512))
    vel[0] = u0 * np.sin(2 * np.pi * (Y + 0.5) / ny) * np.cos(2 * np.pi * (Z + 0.5) / nz)
    vel[1] = u0 * np.cos(2 * np.pi * (X + 0.5) / nx)
    vel[2] = 0.5 * u0 * np.sin(2 * np.pi * (X + Y + 1.0) / nx)
    vel += noise * u0 * rng.standard_normal(vel.shape)
    rho = 1.0 + 0.01 * np.cos(2 * np.pi * (X + 0.5) / nx) + 0.001 * rng.standard_normal((dom.n_blocks, 512))
    return rho, vel


def pair(env, dims, rho, vel):
    oracle, solver = env
    dom = solver.build_box(*dims, periodic=(True, True, True))
    geom = solver.Geometry(dom)
    lvl = solver.Level(geom, "entropic", math="exact")
    lvl.init_equilibrium(rho, vel)
    ora = oracle.OracleQ39Level(dom.neighbor_table).init_equilibrium(rho, vel)
    return dom, geom, lvl, ora


def assert_same_state(lvl, ora):
    f, rho, vel = lvl.state()
    lam = lvl.lambda_cache()
    assert same_bits(f, ora.f), np.abs(f - ora.f).max()
    assert same_bits(vel, ora.vel), np.abs(vel - ora.vel).max()
    assert same_bits(rho, ora.rho), np.abs(rho - ora.rho).max()
    assert same_bits(lam, ora.lam)


def test_init_equilibrium_bitwise(env):
    dom_dims = (2, 1, 1)
    oracle, solver = env
    dom = solver.build_box(*dom_dims, periodic=(True, True, True))
    rho, vel = smooth_fields(dom, u0=0.2)
    _, geom, lvl, ora = pair(env, dom_dims, rho, vel)
    f, r, v = lvl.state()
    assert same_bits(f, ora.f) and same_bits(r, ora.rho) and same_bits(v, ora.vel)
    assert np.all(np.isnan(lvl.lambda_cache()))


CONFIGS = {
    "bisection": dict(tau=0.6, c_wale=0.2),
    "newton": dict(tau=0.52, c_wale=0.2, adaptive_omega4=1),
    "approximate": dict(tau=0.55, adaptive_omega4=2),
    "taylor": dict(tau=0.58, c_wale=0.1, adaptive_omega4=3),
    "sigma_hrr_floors": dict(tau=0.51, c_wale=0.3, lambda_param=0.3, hrr_hybrid=1, hrr_sigma=0.9,
                             nu_sgs_background=0.002, nu_sgs_lattice_floor=0.004),
}


@pytest.mark.parametrize("name", list(CONFIGS))
def test_level_steps_bitwise(env, name):
    oracle, solver = env
    dims = (2, 2, 2)
    dom = solver.build_box(*dims, periodic=(True, True, True))
    rho, vel = smooth_fields(dom, u0=0.08, seed=1)
    _, geom, lvl, ora = pair(env, dims, rho, vel)
    p = solver.default_entropic_params(**CONFIGS[name])
    for _ in range(3):
        lvl.step(p)
        ora.step(p)
    assert_same_state(lvl, ora)


def test_transonic_branches_bitwise(env):
    """|u| above the far-bulk caps and Mach 0.5: macro realizability clamp, equilibrium velocity
    cap, Mach-pocket viscosity and sigma, realizability guards."""
    oracle, solver = env
    dims = (2, 2, 1)
    dom = solver.build_box(*dims, periodic=(True, True, True))
    X, Y, Z = cell_xyz(dom)
    vel = np.zeros((3, dom.n_blocks, 512))
    vel[0] = 0.45 + 0.3 * np.sin(2 * np.pi * (Y + 0.5) / 16)
    vel[1] = 0.45 * np.sin(2 * np.pi * (X + 0.5) / 16)
    vel[2] = 0.1 * np.cos(2 * np.pi * (Z + 0.5) / 8)
    rho = 1.0 + 0.5 * np.sin(2 * np.pi * (X + Y + 1.0) / 16)  # 0.5 .. 1.5: density guards too
    _, geom, lvl, ora = pair(env, dims, rho, vel)
    p = solver.default_entropic_params(tau=0.502, c_wale=0.2, u_inlet=0.45, shock_nu_max=0.02)
    for _ in range(3):
        lvl.step(p)
        ora.step(p)
    assert_same_state(lvl, ora)
    assert np.all(np.isfinite(ora.f))


def test_nan_reset_bitwise(env):
    oracle, solver = env
    dims = (1, 1, 2)
    dom = solver.build_box(*dims, periodic=(True, True, True))
    rho, vel = smooth_fields(dom, u0=0.05, seed=2)
    _, geom, lvl, ora = pair(env, dims, rho, vel)
    f, r, v = lvl.state()
    f[:, 0, 100] = np.nan
    f[:, 1, 300] = 1e-5
    lvl.set_state(f, r, v)
    ora.f[...] = f.astype(np.float32)
    ora.rho[...] = r
    ora.vel[...] = v
    ora.lam[...] = np.nan
    p = solver.default_entropic_params(tau=0.6, u_inlet=0.07)
    for _ in range(2):
        lvl.step(p)
        ora.step(p)
    assert_same_state(lvl, ora)
    assert np.all(np.isfinite(ora.f))


def test_advance_graph_equals_steps(env):
    oracle, solver = env
    dims = (2, 2, 2)
    dom = solver.build_box(*dims, periodic=(True, True, True))
    rho, vel = smooth_fields(dom, u0=0.06, seed=3)
    p = solver.default_entropic_params(tau=0.56, c_wale=0.2)
    geom = solver.Geometry(dom)
    a = solver.Level(geom, "entropic", math="exact")
    b = solver.Level(geom, "entropic", math="exact")
    a.init_equilibrium(rho, vel)
    b.init_equilibrium(rho, vel)
    a.advance(p, 5)
    a.advance(p, 5)
    for _ in range(10):
        b.step(p)
    fa, ra, va = a.state()
    fb, rb, vb = b.state()
    assert same_bits(fa, fb) and same_bits(ra, rb) and same_bits(va, vb)
    assert same_bits(a.lambda_cache(), b.lambda_cache())


def test_lambda_cache_round_trip_and_mass_momentum(env):
    oracle, solver = env
    dims = (1, 2, 1)
    dom = solver.build_box(*dims, periodic=(True, True, True))
    rho, vel = smooth_fields(dom, u0=0.05, seed=4)
    _, geom, lvl, ora = pair(env, dims, rho, vel)
    p = solver.default_entropic_params(tau=0.6)
    lvl.step(p)
    lam = lvl.lambda_cache()
    assert np.all(np.isfinite(lam))
    lam2 = lam.copy()
    lam2[:, 0, :10] = np.nan
    lvl.lambda_cache(lam2)
    assert same_bits(lvl.lambda_cache(), lam2)
    f, _, _ = lvl.state()
    t = oracle.q39_tables()
    c = np.stack([t["cx"], t["cy"], t["cz"]]).astype(np.float64)
    ref = np.array([f.sum(), *np.tensordot(c, f, axes=(1, 0)).sum(axis=(1, 2))])
    assert np.allclose(lvl.mass_momentum(), ref, rtol=1e-12, atol=1e-9)


def test_refused_configurations(env):
    oracle, solver = env
    from openaerolab_alpha_01_b200._capi import OALError
    dom = solver.build_box(2, 2, 2, periodic=(True, True, True))
    geom = solver.Geometry(dom)
    with pytest.raises(OALError):
        solver.Level(geom, "entropic", storage="f16")
    lvl = solver.Level(geom, "entropic", math="exact")
    rho, vel = smooth_fields(dom)
    lvl.init_equilibrium(rho, vel)
    with pytest.raises(OALError):
        lvl.step(solver.default_step_params(tau=0.6))  # cumulant operator id
    with pytest.raises(OALError):
        lvl.step(solver.default_entropic_params(tau=0.6, adaptive_omega4=4))


def test_conservation_and_viscosity_at_scale(env):
    """A 64^3 box with a shear wave (wavelength 64) over a uniform cross flow: FP64 mass holds to
    FP32 round-off (under 2.5e-8 per cell and step); momentum to the 13-moment solve's tolerance
    (its residual stops at 22.5 float eps and the KBC update moves momentum by about twice the
    residual: bound 1e-7 per cell and step); the decay rate gives nu = cs^2 (tau - 1/2) within 3 %.
    The wave decays by a fifth per 100 steps: a slower decay would drown in the solve's FP32
    residual (at wavelength 128, tau 0.7 the same measurement scatters by +-40 % with amplitude)."""
    oracle, solver = env
    dom = solver.build_box(8, 8, 8, periodic=(True, True, True))
    X, Y, Z = cell_xyz(dom)
    L = 64
    k = 2 * np.pi / L
    vel = np.zeros((3, dom.n_blocks, 512))
    vel[0] = 0.03 * np.sin(k * (Y + 0.5))
    vel[2] = 0.01
    rho = np.ones((dom.n_blocks, 512))
    geom = solver.Geometry(dom)
    lvl = solver.Level(geom, "entropic", math="exact")
    lvl.init_equilibrium(rho, vel)
    tau = 0.8
    p = solver.default_entropic_params(tau=tau, c_wale=0.0)
    m0 = lvl.mass_momentum()
    amp = []
    for _ in range(2):
        lvl.advance(p, 100)
        _, _, v = lvl.state()
        amp.append(2 * np.mean(v[0] * np.sin(k * (Y + 0.5))))
    m1 = lvl.mass_momentum()
    n = dom.n_blocks * 512
    assert abs(m1[0] - m0[0]) / (n * 200) < 2.5e-8
    assert np.max(np.abs(m1[1:] - m0[1:])) / (n * 200) < 1e-7
    nu = np.log(amp[0] / amp[1]) / 100 / k ** 2
    assert abs(nu / (CS2 * (tau - 0.5)) - 1) < 0.03, nu


def channel_pair(env, **kw):
    """A 32 x 16 x 16 channel with a sphere (diameter 6): velocity inlet, zero-gradient outlet,
    mirror faces in y and z, full-way bounce-back in the sphere."""
    oracle, solver = env
    from openaerolab_alpha_01_b200.cases import sphere_channel_case
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=12.0, u_inlet=0.05, re=200.0)
    d = case.dom
    geom = solver.Geometry(d)
    lvl = solver.Level(geom, "entropic", math="exact")
    rng = np.random.default_rng(5)
    vel = case.vel + 0.005 * rng.standard_normal(case.vel.shape) * (d.obstacle == 0)
    lvl.init_equilibrium(case.rho, vel)
    ora = oracle.OracleQ39Level(d.neighbor_table, d.coords, d.shape, d.obstacle).init_equilibrium(case.rho, vel)
    p = solver.default_entropic_params(tau=0.56, c_wale=0.2, u_inlet=0.05, **kw)
    return d, geom, lvl, ora, p


FACE_CONFIGS = {
    "faces": dict(),
    "inlet_noise": dict(inlet_turbulence=0.05),
    "ground_wall": dict(ymin_wall_bc=1),
    "transverse_freestream": dict(transverse_freestream=1, transverse_freestream_blend=0.3),
}


@pytest.mark.parametrize("name", list(FACE_CONFIGS))
def test_channel_faces_and_obstacle_bitwise(env, name):
    """Domain faces (inlet with its mass/momentum pin, outlet, mirrors, ground, transverse
    freestream, inlet noise) and the obstacle's bounce-back: the oracle's bits after 4 steps."""
    d, geom, lvl, ora, p = channel_pair(env, **FACE_CONFIGS[name])
    for i in range(4):
        p.time_step_seed = 7 + i
        lvl.step(p)
        ora.step(p)
    assert_same_state(lvl, ora)
    _, _, v = lvl.state()
    assert np.all(v[:, d.obstacle.astype(bool)] == 0.0)
    assert np.all(np.isfinite(ora.f))


@pytest.mark.parametrize("blend", [0, 1])
def test_channel_sponge_and_near_wall_bitwise(env, blend):
    """The sponge toward the inlet state (with and without the population blend) and the near-wall
    bounds of the macro realizability clamp (wall distance under 16 cells around the sphere and
    the sponge strips): the oracle's bits after 4 steps, on a state pushed into the clamp."""
    oracle, solver = env
    from openaerolab_alpha_01_b200.cases import sphere_channel_case
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=12.0, u_inlet=0.05, re=200.0)
    d = case.dom
    gx, gy, gz = d.cell_positions()
    d.sponge = (np.clip((gx - 24.0) / 8.0, 0.0, 1.0) * 0.6).astype(np.float32)
    r = np.sqrt((gx - 0.5 - 12.0) ** 2 + (gy - 0.5 - 8.0) ** 2 + (gz - 0.5 - 8.0) ** 2) - 3.0
    d.wall_dist = np.where(d.obstacle != 0, 0.0, np.maximum(r, 0.0)).astype(np.float32)
    geom = solver.Geometry(d)
    lvl = solver.Level(geom, "entropic", math="exact")
    rng = np.random.default_rng(7)
    vel = case.vel + 0.005 * rng.standard_normal(case.vel.shape) * (d.obstacle == 0)
    rho = case.rho.copy()
    # a dense pocket near the sphere and a fast one in the far field: both clamp branches fire
    rho[(r > 0) & (r < 3)] = 2.3
    vel[0][(r > 10) & (gx < 24)] = 0.7
    lvl.init_equilibrium(rho, vel)
    ora = oracle.OracleQ39Level(d.neighbor_table, d.coords, d.shape, d.obstacle, sponge=d.sponge,
                                wall_dist=d.wall_dist).init_equilibrium(rho, vel)
    p = solver.default_entropic_params(tau=0.56, c_wale=0.2, u_inlet=0.05, sponge_blend_distributions=blend)
    for i in range(4):
        p.time_step_seed = 11 + i
        lvl.step(p)
        ora.step(p)
    assert_same_state(lvl, ora)
    assert np.all(np.isfinite(ora.f))


def test_channel_advance_graph_equals_steps(env):
    """n steps in one graph advance the noise seed by one per step, as single steps do."""
    d, geom, a, _, p = channel_pair(env, inlet_turbulence=0.05)
    oracle, solver = env
    b = solver.Level(geom, "entropic", math="exact")
    fa, ra, va = a.state()
    b.set_state(fa, ra, va)
    p.time_step_seed = 3
    a.advance(p, 4)
    for i in range(4):
        q = solver.default_entropic_params(tau=0.56, c_wale=0.2, u_inlet=0.05, inlet_turbulence=0.05)
        q.time_step_seed = 3 + i
        b.step(q)
    fa, ra, va = a.state()
    fb, rb, vb = b.state()
    assert same_bits(fa, fb) and same_bits(ra, rb) and same_bits(va, vb)


# The default math of a D3Q39 level (CUDA's expf / logf, the cached multipliers accepted as the
# solve's start up to a moment residual of ~3e-2): the same step within tolerance of the oracle.
# Bounds after 3 steps, relative to the field's maximum: populations and velocity 2e-3, density
# 2e-4 (the entropic alpha solvers turn ulp-level exp/log differences into differences of the
# alpha root within its 0.5 % bisection tolerance; the Newton solver is the most sensitive).
@pytest.mark.parametrize("name", list(CONFIGS))
def test_fast_math_within_tolerance(env, name):
    oracle, solver = env
    dims = (2, 2, 2)
    dom = solver.build_box(*dims, periodic=(True, True, True))
    rho, vel = smooth_fields(dom, u0=0.08, seed=1)
    geom = solver.Geometry(dom)
    lvl = solver.Level(geom, "entropic")
    lvl.init_equilibrium(rho, vel)
    ora = oracle.OracleQ39Level(dom.neighbor_table).init_equilibrium(rho, vel)
    p = solver.default_entropic_params(**CONFIGS[name])
    for _ in range(3):
        lvl.step(p)
        ora.step(p)
    f, r, v = lvl.state()
    lam = lvl.lambda_cache()

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    assert rel(f, ora.f) < 2e-3
    assert rel(v, ora.vel) < 2e-3
    assert rel(r, ora.rho) < 2e-4
    assert np.array_equal(np.isnan(lam), np.isnan(ora.lam))
    fin = np.isfinite(lam)
    assert float(np.max(np.abs(lam[fin] - ora.lam[fin])) / np.max(np.abs(ora.lam[fin]))) < 2e-3
