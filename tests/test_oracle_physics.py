"""Physics gates of the CPU oracle, restated from the reference's octree tests
(tools/tests/q19_octree_step.jl): rest state (G0.3), conservation (G0.4), Taylor-Green decay and
order (G1.2); plus a regression fixture of the oracle on a small sphere channel and planted-mistake
checks that show the comparisons are sensitive."""
import json
from pathlib import Path

import numpy as np
import pytest

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200.solver import BlockDomain, kinetic_energy, taylor_green_fields

GOLDEN = Path(__file__).resolve().parent / "golden"


def params(**kw):
    return capi.default_params(**kw)


def periodic(oracle, n, dtype=np.float64):
    coords, nbr = oracle.build_box(n // 8, n // 8, n // 8, 7)
    return coords, nbr, oracle.OracleLevel(coords, nbr, (n, n, n), dtype=dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_rest_state_stays_at_rest(oracle_lib, dtype):
    """G0.3 analogue: the octree's shifted populations keep the rest state exactly; the cumulant
    moments of w_k are not exact in binary, so the D3Q27 state must stay within a few ulps."""
    coords, nbr, L = periodic(oracle_lib, 16, dtype)
    nb = coords.shape[0]
    L.init_equilibrium(np.ones((nb, 512)), np.zeros((3, nb, 512)))
    f0 = L.f.copy()
    p = params(tau=0.52)
    for _ in range(20):
        L.step(p)
    eps = np.finfo(dtype).eps
    assert np.max(np.abs(L.f - f0)) <= 8 * eps
    assert np.max(np.abs(L.vel)) <= 8 * eps


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-6)])
def test_conservation(oracle_lib, dtype, tol):
    coords, nbr, L = periodic(oracle_lib, 16, dtype)
    dom = BlockDomain(2, 2, 2, coords, nbr)
    gx, gy, gz = dom.cell_positions()
    x, y, z = gx - 0.5, gy - 0.5, gz - 0.5
    rho = 1.0 + 0.01 * np.sin(2 * np.pi * x / 16) * np.cos(2 * np.pi * z / 16)
    vel = np.stack([0.03 * np.sin(2 * np.pi * y / 16), 0.02 * np.cos(2 * np.pi * z / 16),
                    0.01 * np.sin(2 * np.pi * x / 16)])
    L.init_equilibrium(rho, vel)
    m0 = L.mass_momentum()
    p = params(tau=0.52, c_wale=0.2)
    for _ in range(50):
        L.step(p)
    m1 = L.mass_momentum()
    assert abs(m1[0] - m0[0]) / m0[0] < tol
    assert np.max(np.abs(m1[1:] - m0[1:])) / (16 ** 3 * 0.03) < tol
    assert np.all(np.isfinite(L.f))


def tgv_error(oracle, n, nu=0.01, u0=0.01):
    coords, nbr, L = periodic(oracle, n)
    dom = BlockDomain(n // 8, n // 8, n // 8, coords, nbr)
    rho, vel = taylor_green_fields(dom, u0)
    L.init_equilibrium(rho, vel)
    p = params(tau=3 * nu + 0.5, c_wale=0.0)
    steps = 125 * (n // 16) ** 2
    s1 = steps // 5
    for _ in range(s1):
        L.step(p)
    ke1 = kinetic_energy(L.rho, L.vel)
    for _ in range(steps - s1):
        L.step(p)
    ke2 = kinetic_energy(L.rho, L.vel)
    k = 2 * np.pi / n
    expected = np.exp(-4 * nu * k * k * (steps - s1))
    return abs(ke2 / ke1 - expected) / expected


def test_taylor_green_order(oracle_lib):
    e16 = tgv_error(oracle_lib, 16)
    e32 = tgv_error(oracle_lib, 32)
    assert e32 < 0.01
    assert np.log(e16 / e32) / np.log(2) >= 1.8


def _channel_case(oracle):
    from tests.golden.make_golden import channel_case
    return channel_case(oracle)


def test_oracle_regression_fixture(oracle_lib):
    """The oracle reproduces its committed fixture (sphere channel, half-way walls, FP64)."""
    ref = json.loads((GOLDEN / "oracle_channel_fp64.json").read_text())
    out = _channel_case(oracle_lib)
    assert out["n_solid"] == ref["n_solid"]
    for key in ("force", "mass_momentum"):
        np.testing.assert_allclose(out[key], ref[key], rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(out["probe_f"], ref["probe_f"], rtol=1e-11, atol=1e-14)


def test_planted_mistakes_are_detected(oracle_lib):
    """Changing one relaxation rate or the limiter moves the state far beyond the parity
    tolerances used against the CUDA path (1e-9 FP64, 2e-5 FP32)."""
    coords, nbr, A = periodic(oracle_lib, 16)
    _, _, B = periodic(oracle_lib, 16)
    dom = BlockDomain(2, 2, 2, coords, nbr)
    rho, vel = taylor_green_fields(dom, 0.05)
    A.init_equilibrium(rho, vel)
    B.init_equilibrium(rho, vel)
    pa = params(tau=0.51, c_wale=0.2)
    pb = params(tau=0.51, c_wale=0.2, omega3=0.99)
    for _ in range(10):
        A.step(pa)
        B.step(pb)
    rel = np.max(np.abs(A.f - B.f)) / np.max(np.abs(A.f))
    assert rel > 1e-7


def test_grad_wall_properties(oracle_lib):
    """The Grad-reconstruction wall (bc_scheme "grad", geometry/grad_wall_kernel.jl): every fluid
    cell with a link into the sphere leaves the step with zero velocity output, populations of
    the rebuilt form rho w_k + (1 - 1/tau) w_k 4.5 Q_k : Pi (so each cell keeps its density and
    carries zero momentum), at least 1e-12; with grad_pineq_scale 0 the wall cells hold exactly
    the rest equilibrium rho w_k. Cells away from the wall step as with the full-way treatment."""
    from openaerolab_alpha_01_b200 import _capi as capi
    from openaerolab_alpha_01_b200.cases import sphere_channel_case
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=12.0, u_inlet=0.05, re=200.0)
    d = case.dom
    k = np.arange(27)
    c = np.stack([k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1]).astype(np.float64)
    w = np.array([{0: 8 / 27, 1: 2 / 27, 2: 1 / 54, 3: 1 / 216}[int(v)] for v in (c * c).sum(0)])

    def run(bc, scale=1.0, steps=3):
        O = oracle_lib.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle, dtype=np.float64)
        O.init_equilibrium(case.rho, case.vel)
        p = capi.default_params(**{f: getattr(case.params, f) for f, _ in capi.StepParams._fields_ if f != "reserved"})
        p.solid_bc, p.collect_forces, p.grad_pineq_scale = bc, 0, scale
        for i in range(steps):
            p.time_step_seed = i
            O.step(p)
        return O
    # fluid cells with a solid pull source
    solid = d.obstacle.astype(bool)
    X, Y, Z = d.cell_positions()
    sx, sy, sz = d.shape
    occ = np.zeros((sx + 2, sy + 2, sz + 2), bool)
    occ[X[solid], Y[solid], Z[solid]] = True
    wall = np.zeros_like(solid)
    for q in range(27):
        wall |= occ[X - c[0, q].astype(int), Y - c[1, q].astype(int), Z - c[2, q].astype(int)]
    wall &= ~solid
    assert wall.sum() > 50
    G = run(capi.OAL_SOLID_GRAD)
    F = run(capi.OAL_SOLID_FULLWAY)
    assert np.all(G.vel[:, wall] == 0.0)
    fw = G.f[:, wall]                                   # (27, n_wall)
    assert np.all(fw >= 1e-12)
    rho = fw.sum(0)
    assert np.allclose(rho, G.rho[wall], rtol=1e-12)
    assert np.max(np.abs(c @ fw)) < 1e-13
    G0 = run(capi.OAL_SOLID_GRAD, scale=0.0, steps=1)
    assert np.allclose(G0.f[:, wall], w[:, None] * G0.rho[wall][None, :], rtol=1e-13, atol=0)
    # away from the wall (two cells or more from any wall cell after three steps) nothing differs
    far = ~solid & ~wall
    for _ in range(3):
        grown = far.copy()
        occ2 = np.ones((sx + 2, sy + 2, sz + 2), bool)
        occ2[X[~far], Y[~far], Z[~far]] = False
        for q in range(27):
            grown &= occ2[X - c[0, q].astype(int), Y - c[1, q].astype(int), Z - c[2, q].astype(int)]
        far = grown
    assert far.sum() > 1000
    assert np.array_equal(G.f[:, far], F.f[:, far])
