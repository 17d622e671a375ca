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
