"""Variable eddy viscosity of the oracle's D3Q27 step (kernel_cumulant.jl:546-588,
kernel_dynamic_sgs.jl:124-240, kernel_pi_neq.jl:39-180), on the CPU.

* a uniform stream has no strain: both modes reduce to the floor, which is the background path
  with nu_sgs_background = floor, bit for bit;
* a constant stored Pi_neq gives nu_sgs = c_pi |tau / (tau - 1)| |Pi| / (rho cs^2), the same step
  as the background path with that value;
* the refreshed field equals the Pi_neq of the stored state, bit for bit (the refresh is the
  diagnostic evaluated on the step's outputs);
* Pi_neq of an equilibrium state is zero, and Pi_neq is zero in solid cells.
"""
import numpy as np
import pytest

from openaerolab_alpha_01_b200.cases import sphere_channel_case, taylor_green_case


def uniform_case(oracle, n=2, u=(0.03, -0.01, 0.02)):
    coords, nbr = oracle.build_box(n, n, n, 7)
    nb = coords.shape[0]
    rho = np.ones((nb, 512))
    vel = np.zeros((3, nb, 512))
    for c in range(3):
        vel[c] = u[c]
    return coords, nbr, (8 * n, 8 * n, 8 * n), rho, vel


def params(oracle, **kw):
    p = oracle.default_step_params()
    p.tau = 0.56
    p.u_inlet = 0.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("mode", [1, 2])
def test_uniform_stream_reduces_to_the_floor(oracle_lib, mode):
    coords, nbr, shape, rho, vel = uniform_case(oracle_lib)
    runs = []
    for p in (params(oracle_lib, variable_nu_sgs=mode, nu_sgs_floor=0.004),
              params(oracle_lib, nu_sgs_background=0.004)):
        O = oracle_lib.OracleLevel(coords, nbr, shape, dtype=np.float64)
        O.init_equilibrium(rho, vel)
        # a small perturbation of the populations (not of the macros' uniformity) so that the
        # collision does work; the strain stays zero
        O.f *= 1.0 + 1e-3 * np.cos(np.arange(27))[:, None, None]
        for _ in range(3):
            O.step(p)
        runs.append(O.f.copy())
    assert np.array_equal(runs[0], runs[1])


def test_pi_stress_viscosity_closed_form(oracle_lib):
    coords, nbr, shape, rho, vel = uniform_case(oracle_lib)
    tau, c_pi, a = 0.56, 0.2, 3e-3
    pert = 1.0 + 1e-3 * np.sin(np.arange(27))[:, None, None]
    O = oracle_lib.OracleLevel(coords, nbr, shape, dtype=np.float64)
    O.init_equilibrium(rho, vel)
    rho_cell = float(np.sum(O.f[:, 0, 0] * pert[:, 0, 0]))  # the perturbed cells' density
    nu_s = c_pi * abs(tau / (tau - 1.0)) * a / (rho_cell / 3.0 + 1e-10)
    out = []
    # nu_sgs_background is a float parameter: the two paths differ by its rounding (~6e-8 of nu_s)
    for p in (params(oracle_lib, tau=tau, variable_nu_sgs=1, c_pi=c_pi, nu_sgs_floor=0.0),
              params(oracle_lib, tau=tau, nu_sgs_background=nu_s, c_wale=0.0),
              params(oracle_lib, tau=tau, nu_sgs_background=0.0, c_wale=0.0)):
        O = oracle_lib.OracleLevel(coords, nbr, shape, dtype=np.float64)
        O.init_equilibrium(rho, vel)
        O.f *= pert
        O.pi_neq[0] = a  # |Pi| = a (xx only)
        O.step(p)
        out.append(O.f.copy())
    assert nu_s > 1e-3
    scale = np.max(np.abs(out[1]))
    d_model, d_none = np.max(np.abs(out[0] - out[1])), np.max(np.abs(out[0] - out[2]))
    assert d_none > 1e-7 * scale
    assert d_model < 1e-5 * d_none


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_refreshed_field_is_the_state_pi_neq(oracle_lib, dtype):
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    d = case.dom
    O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, sponge=d.sponge,
                               wall_dist=d.wall_dist, dtype=dtype)
    O.init_equilibrium(case.rho, case.vel)
    p = case.params
    p.variable_nu_sgs = 1
    p.nu_sgs_floor = 0.0
    for _ in range(6):
        O.step(p)
    ref = O.state_pi_neq()
    if dtype == np.float64:
        assert np.array_equal(O.pi_neq, ref)
    else:
        # float refresh against the double evaluation: Pi_neq is a difference of O(rho cs^2) sums,
        # so its float error is absolute, a few ulp of 1/3
        assert np.max(np.abs(O.pi_neq - ref)) < 2e-7
    assert np.all(O.pi_neq[:, d.obstacle == 1] == 0)
    assert np.max(np.abs(ref)) > 1e-6


def test_equilibrium_state_has_no_pi_neq(oracle_lib):
    case = taylor_green_case(16, u0=0.05, re=100.0)
    d = case.dom
    O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, dtype=np.float64)
    O.init_equilibrium(case.rho, case.vel)
    assert np.max(np.abs(O.state_pi_neq())) < 1e-15


def test_dynamic_mode_sees_strain(oracle_lib):
    """On a Taylor-Green vortex the dynamic coefficient is non-zero somewhere: with the floor at
    zero and WALE off, the step differs from a plain step."""
    case = taylor_green_case(16, u0=0.08, re=200.0)
    d = case.dom
    fs = []
    for mode in (0, 2):
        O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, dtype=np.float64)
        O.init_equilibrium(case.rho, case.vel)
        p = case.params
        p.c_wale = 0.0
        p.variable_nu_sgs = mode
        p.nu_sgs_floor = 0.0
        for _ in range(4):
            O.step(p)
        fs.append(O.f.copy())
    assert np.max(np.abs(fs[0] - fs[1])) > 1e-9
