"""Spectral vanishing viscosity of the oracle (kernel_svv_yz_d3q39.jl), on the CPU.

D3Q27 post-pass (apply_svv_d3q19_postcollision!, :426-458, with apply_svv_d3q19_inline!):
* a shear-stress checkerboard of zero mass and momentum is the bi-Laplacian's eigenmode: one pass
  scales it by 1 - 16 eps per filtered axis at Nyquist, in closed form;
* the 4-moment correction keeps every cell's mass and momentum;
* the taps' fall-backs (a solid cell, a missing neighbour block: the cell's own input population)
  agree with a plain-Python restatement of get_pop_neighbor_x / _yz (:78-116, 225-250);
* the strengths of a level are gated by its level number as timestep.jl:1577-1578 gates them.
D3Q39 (inside the KBC step, kernel_entropic_d3q39.jl:3256-3318): the filter leaves the step's
mass and momentum alone and damps a checkerboard the step alone keeps.
"""
import numpy as np
import pytest

FLOOR = float(np.float32(1e-12))  # the population floor, a binary32 constant widened

from openaerolab_alpha_01_b200.cases import taylor_green_case
from openaerolab_alpha_01_b200.solver import svv_epsilons


def checkerboard_state(oracle, axis, amp=2e-3):
    """f_k = w_k (1 + amp c_x c_y (-1)^i) on a periodic 2 x 2 x 2 box, i the cell index along
    `axis` (0 x, 1 y, 2 z, 3 y + z): mass and momentum are uniform, Pi_xy alternates."""
    t = oracle.d3q27_tables()
    coords, nbr = oracle.build_box(2, 2, 2, 7)
    nb = coords.shape[0]
    cell = np.arange(512)
    lx, ly, lz = cell % 8, (cell // 8) % 8, cell // 64
    gx = (coords[:, 0:1] - 1) * 8 + lx
    gy = (coords[:, 1:2] - 1) * 8 + ly
    gz = (coords[:, 2:3] - 1) * 8 + lz
    i = [gx, gy, gz, gy + gz][axis]
    sign = np.where(i % 2 == 0, 1.0, -1.0)
    w, cx, cy = t["w"], t["cx"].astype(float), t["cy"].astype(float)
    f = w[:, None, None] * (1.0 + amp * (cx * cy)[:, None, None] * sign[None])
    return t, coords, nbr, nb, np.ascontiguousarray(f), sign


@pytest.mark.parametrize("axis,eps_x,eps_yz,n_axes", [
    (1, 0.0, 0.004, 1),   # y Nyquist, y-z filter
    (2, 0.0, 0.004, 1),   # z Nyquist, y-z filter
    (3, 0.0, 0.004, 2),   # (-1)^(y+z): both axes
    (0, 0.003, 0.0, 1),   # x Nyquist, x filter
    (0, 0.0, 0.004, 0),   # x Nyquist is outside the y-z filter
    (1, 0.003, 0.0, 0),   # and y Nyquist outside the x filter
])
def test_shear_checkerboard_closed_form(oracle_lib, axis, eps_x, eps_yz, n_axes):
    t, coords, nbr, nb, f, sign = checkerboard_state(oracle_lib, axis)
    f_out = f.copy()
    oracle_lib.svv_d3q27(nb, nbr, None, eps_x, eps_yz, f, f_out)
    eps = float(np.float32(max(eps_x, eps_yz)))   # the strengths are binary32 parameters
    factor = 1.0 - 16.0 * n_axes * eps
    w, cx, cy = t["w"], t["cx"].astype(float), t["cy"].astype(float)
    expect = w[:, None, None] * (1.0 + factor * 2e-3 * (cx * cy)[:, None, None] * sign[None])
    assert np.max(np.abs(f_out - expect)) < 1e-16


def test_mass_and_momentum_of_every_cell_kept(oracle_lib):
    case = taylor_green_case(16, u0=0.05, re=400.0)
    t = oracle_lib.d3q27_tables()
    coords, nbr = oracle_lib.build_box(2, 2, 2, 0)  # no periodic axis: the domain-edge fall-back
    nb = coords.shape[0]
    obst, n_solid = oracle_lib.sphere(coords, (8.0, 8.0, 8.0), 3.0)
    assert n_solid > 0
    rng = np.random.default_rng(3)
    f_in = oracle_lib.init_feq(case.rho, case.vel, 0) * (1 + 1e-2 * rng.standard_normal((27, nb, 512)))
    f_out = oracle_lib.init_feq(case.rho, case.vel, 0) * (1 + 1e-2 * rng.standard_normal((27, nb, 512)))
    f_in, f_out = np.ascontiguousarray(f_in), np.ascontiguousarray(f_out)
    before = f_out.copy()
    oracle_lib.svv_d3q27(nb, nbr, obst, 0.002, 0.004, f_in, f_out)
    c = np.stack([t["cx"], t["cy"], t["cz"]]).astype(float)
    fluid = obst == 0
    assert not np.array_equal(f_out[:, fluid], before[:, fluid])
    assert np.array_equal(f_out[:, ~fluid], before[:, ~fluid])      # solid cells untouched
    for m in (np.ones(27), *c):
        d = np.tensordot(m, f_out - before, axes=(0, 0))
        assert np.max(np.abs(d[fluid])) < 1e-15


def python_svv(nb, nbr, obst, eps_x, eps_yz, f_in, f_out, t):
    """The post-pass written out with the tap helpers' rules, cell by cell."""
    out = f_out.copy()
    cx, cy, cz, w = t["cx"], t["cy"], t["cz"], t["w"]
    eps_x, eps_yz = float(np.float32(eps_x)), float(np.float32(eps_yz))

    def solid(b, x, y, z):
        return obst is not None and obst[b, x + 8 * y + 64 * z] != 0

    def tap(b, x, y, z, d, k):
        n = [x + d[0], y + d[1], z + d[2]]
        o = [-1 if v < 0 else (1 if v > 7 else 0) for v in n]
        own = f_in[k, b, x + 8 * y + 64 * z]
        if o == [0, 0, 0]:
            return own if solid(b, *n) else f_in[k, b, n[0] + 8 * n[1] + 64 * n[2]]
        nbb = nbr[(o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1), b]
        if nbb == 0:
            return own
        ln = [v - 8 * s for v, s in zip(n, o)]
        if solid(nbb - 1, *ln):
            return own
        return f_in[k, nbb - 1, ln[0] + 8 * ln[1] + 64 * ln[2]]

    for b in range(nb):
        for cell in range(512):
            x, y, z = cell % 8, (cell // 8) % 8, cell // 64
            if solid(b, x, y, z):
                continue
            fl = [0.0] * 27
            dr = dx = dy = dz = 0.0
            for k in range(27):
                fc = f_out[k, b, cell]
                bl = 0.0
                if eps_x > 0:
                    T = lambda s: tap(b, x, y, z, (s, 0, 0), k)
                    bl += eps_x * (T(-2) - 4.0 * T(-1) + 6.0 * fc - 4.0 * T(1) + T(2))
                if eps_yz > 0:
                    T = lambda s: tap(b, x, y, z, (0, s, 0), k)
                    bl += eps_yz * (T(-2) - 4.0 * T(-1) + 6.0 * fc - 4.0 * T(1) + T(2))
                    T = lambda s: tap(b, x, y, z, (0, 0, s), k)
                    bl += eps_yz * (T(-2) - 4.0 * T(-1) + 6.0 * fc - 4.0 * T(1) + T(2))
                ff = fc - bl
                diff = ff - fc
                dr += diff
                dx += diff * float(cx[k]); dy += diff * float(cy[k]); dz += diff * float(cz[k])
                fl[k] = ff
            for k in range(27):
                cu = float(cx[k]) * dx + float(cy[k]) * dy + float(cz[k]) * dz
                v = fl[k] - float(w[k]) * (dr + (1.0 / (1.0 / 3.0)) * cu)
                out[k, b, cell] = FLOOR if v < FLOOR else v
    return out


def test_taps_match_a_plain_restatement(oracle_lib):
    t = oracle_lib.d3q27_tables()
    coords, nbr = oracle_lib.build_box(2, 1, 1, 2)   # y periodic, x and z open
    nb = coords.shape[0]
    obst, n_solid = oracle_lib.sphere(coords, (8.0, 4.0, 3.0), 2.5)
    assert n_solid > 0
    rng = np.random.default_rng(5)
    w = t["w"][:, None, None]
    f_in = np.ascontiguousarray(w * (1 + 0.05 * rng.standard_normal((27, nb, 512))))
    f_out = np.ascontiguousarray(w * (1 + 0.05 * rng.standard_normal((27, nb, 512))))
    got = f_out.copy()
    oracle_lib.svv_d3q27(nb, nbr, obst, 0.003, 0.005, f_in, got)
    ref = python_svv(nb, nbr, obst, 0.003, 0.005, f_in, f_out, t)
    assert np.array_equal(got, ref)


def test_floor_and_post_copy(oracle_lib):
    t, coords, nbr, nb, f, _ = checkerboard_state(oracle_lib, 1)
    f_out = f.copy()
    f_out[5, 0, 17] = -1e-3                     # a negative post-collision population
    post = np.zeros_like(f_out)
    oracle_lib.svv_d3q27(nb, nbr, None, 0.0, 0.002, f, f_out, post)
    assert f_out.min() >= FLOOR and f_out[5, 0, 17] == FLOOR
    assert np.array_equal(post, f_out)


def test_level_gating():
    assert svv_epsilons(1) == dict(svv_yz_epsilon=0.0, svv_x_epsilon=0.0)
    on = dict(yz_enabled=True, x_enabled=True)
    assert svv_epsilons(1, **on) == dict(svv_yz_epsilon=0.0, svv_x_epsilon=0.002)
    assert svv_epsilons(4, **on) == dict(svv_yz_epsilon=0.002, svv_x_epsilon=0.0)
    assert svv_epsilons(2, yz_enabled=True, yz_min_level=2, yz_epsilon=0.01) == dict(svv_yz_epsilon=0.01,
                                                                                       svv_x_epsilon=0.0)
    with pytest.raises(ValueError):
        svv_epsilons(1, yz_min_level=0)


def test_level_step_with_svv_keeps_mass(oracle_lib):
    """The step followed by the filter has the step's mass and momentum (per cell conservation)."""
    case = taylor_green_case(16, u0=0.05, re=400.0)
    runs = []
    for eps in (0.0, 0.004):
        O = oracle_lib.OracleLevel(case.dom.coords, case.dom.neighbor_table, case.dom.shape, dtype=np.float64)
        O.init_equilibrium(case.rho, case.vel)
        p = oracle_lib.default_step_params(tau=case.params.tau, u_inlet=0.0, svv_yz_epsilon=eps, svv_x_epsilon=eps / 2)
        for _ in range(3):
            O.step(p)
        runs.append((O.mass_momentum(), O.f.copy()))
    # the step alone drifts by ~1e-9 at this tau; the filter adds nothing measurable
    assert np.allclose(runs[0][0], runs[1][0], rtol=0, atol=1e-8)
    assert not np.array_equal(runs[0][1], runs[1][1])


# ---- D3Q39 ------------------------------------------------------------------------------------

def q39_box(oracle, n=2):
    coords, nbr = oracle.build_box(n, n, n, 7)
    return coords, nbr, coords.shape[0]


def q39_params(**kw):
    from openaerolab_alpha_01_b200 import solver
    return solver.default_entropic_params(**dict(dict(tau=0.52, u_inlet=0.0, c_wale=0.0), **kw))


def test_q39_svv_keeps_mass_and_damps_a_checkerboard(oracle_lib):
    t = oracle_lib.q39_tables()
    coords, nbr, nb = q39_box(oracle_lib)
    cell = np.arange(512)
    gy = (coords[:, 1:2] - 1) * 8 + (cell // 8) % 8
    sign = np.where(gy % 2 == 0, 1.0, -1.0).astype(np.float32)
    rho = np.ones((nb, 512), np.float32)
    vel = np.zeros((3, nb, 512), np.float32)
    vel[0] = 0.02
    out = {}
    for eps in (0.0, 0.01):
        O = oracle_lib.OracleQ39Level(nbr)
        O.init_equilibrium(rho, vel)
        # a shear-stress checkerboard along y of zero mass and momentum
        cx, cy = t["cx"].astype(np.float32), t["cy"].astype(np.float32)
        O.f += (2e-3 * t["w"] * cx * cy).astype(np.float32)[:, None, None] * sign[None]
        mm0 = O.mass_momentum()
        O.step(q39_params(svv_yz_epsilon=eps))
        mm1 = O.mass_momentum()
        pxy = np.tensordot((cx * cy).astype(np.float64), O.f.astype(np.float64), axes=(0, 0))
        out[eps] = (mm0, mm1, float(np.abs((pxy * sign).mean())))
    for eps, (mm0, mm1, _) in out.items():
        assert np.allclose(mm0, mm1, rtol=0, atol=1e-6 * nb * 512)
    assert out[0.01][2] < out[0.0][2] * 0.95
