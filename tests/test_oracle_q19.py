"""The D3Q19 octree oracle against the reference's own checks (CPU, no GPU).

Known answers restated from the reference's tests:
  tools/tests/q19_kernel.jl:46-75   closed form vs the per-direction collision (2000 random states,
                                    FP64 2e-15, FP32 1e-6), moments and equilibrium vs definitions,
                                    conservation of the collision
  tools/tests/q19_kernel.jl:106-116 pull tables of an oct
  tools/tests/q19_octree_step.jl:30-54  G0.3 rest state exactly zero; G0.4 conservation
The reference's random states come from Julia's generator seeded 20261114; here numpy's generator
with the same seed draws states of the same distribution.
"""
import ctypes as C

import numpy as np
import pytest

SEED = 20261114


def feq_shifted(t, rho, u, dt):
    w = t["w"].astype(dt)
    c = np.stack([t["cx"], t["cy"], t["cz"]]).astype(dt)
    cu = u @ c
    usq = (u * u).sum(-1)
    return (w * rho[:, None] * (dt(1) + dt(3) * cu + dt(4.5) * cu * cu - dt(1.5) * usq[:, None]) - w).astype(dt)


def random_states(t, n, dt, rng, noise=1e-3):
    rho = (0.95 + 0.1 * rng.random(n)).astype(dt)
    u = (0.2 * (rng.random((n, 3)) - 0.5)).astype(dt)
    return (feq_shifted(t, rho, u, dt) + (noise * t["w"][None, :] * rng.standard_normal((n, 19))).astype(dt)).astype(dt)


def kat_inputs(t, dt, n=2000, seed=SEED):
    """The random collision inputs of the closed-form test (q19_kernel.jl:46-60)."""
    rng = np.random.default_rng(seed)
    f = random_states(t, n, dt, rng)
    trial = np.arange(1, n + 1)
    omega = (0.6 + 1.39 * rng.random(n)).astype(dt)
    sigma = np.where(trial % 3 == 0, 1.0, 0.9 + 0.1 * rng.random(n)).astype(dt)
    pfd = (1e-4 * rng.standard_normal((n, 6))).astype(dt)
    F = np.where((trial % 4 == 0)[:, None], 1e-4 * rng.standard_normal((n, 3)), 0.0).astype(dt)
    return f, omega, sigma, pfd, F


def collide_each(oracle, f, omega, sigma, pfd, F, reference=False):
    """sigma is a scalar argument of the collision: call once per distinct sigma."""
    n = f.shape[0]
    out = np.zeros_like(f)
    rho = np.zeros(n, f.dtype)
    u = np.zeros((n, 3), f.dtype)
    for s in np.unique(sigma):
        m = sigma == s
        r = oracle.q19_collide(f[m], omega[m], float(s), pfd[m], F[m], reference=reference)
        if reference:
            out[m] = r
        else:
            out[m], rho[m], u[m] = r
    return (out, rho, u) if not reference else out


@pytest.fixture(scope="module")
def q19(oracle_lib):
    return oracle_lib, oracle_lib.q19_tables()


def test_tables(q19):
    oracle, t = q19
    c = np.stack([t["cx"], t["cy"], t["cz"]])
    assert c.shape == (3, 19) and abs(t["w"].sum() - 1) < 1e-15
    # opposite directions are adjacent pairs (lattice.jl:4-5)
    for i in range(1, 19, 2):
        assert (c[:, i] == -c[:, i + 1]).all()
    # second-moment isotropy: sum w c_a c_b = delta_ab / 3
    m2 = (t["w"][None, None] * c[:, None] * c[None, :]).sum(-1)
    assert np.allclose(m2, np.eye(3) / 3, atol=1e-16)
    # pull tables (q19_kernel.jl:106-112): slot k pulls direction J from slot (x,y,z) - c_J
    for k in range(8):
        x, y, z = k & 1, (k >> 1) & 1, (k >> 2) & 1
        for j in range(19):
            p = np.array([x, y, z]) - c[:, j]
            o = np.clip(np.where(p < 0, -1, np.where(p > 1, 1, 0)), -1, 1)
            assert t["src_off"][k, j] == (o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1)
            q = p - 2 * o
            assert t["src_child"][k, j] == q[0] + 2 * q[1] + 4 * q[2]


@pytest.mark.parametrize("dt,tol", [(np.float64, 2e-15), (np.float32, 1e-6)])
def test_closed_form_against_per_direction(q19, dt, tol):
    """q19_kernel.jl:46-75: the closed-form collision equals the per-direction formulas."""
    oracle, t = q19
    f, omega, sigma, pfd, F = kat_inputs(t, dt)
    out, rho, u = collide_each(oracle, f, omega, sigma, pfd, F)
    ref = collide_each(oracle, f, omega, sigma, pfd, F, reference=True)
    worst = np.abs(out.astype(np.float64) - ref.astype(np.float64)).max()
    assert worst < tol, worst
    # density and velocity of the collision against their definitions
    eps = np.finfo(dt).eps
    drho = f.astype(np.float64).sum(1)
    assert np.abs(rho - 1 - drho).max() < 20 * eps
    forced = (F != 0).any(1)
    m = f.astype(np.float64) @ np.stack([t["cx"], t["cy"], t["cz"]]).T.astype(np.float64)
    uexp = (m + np.where(forced[:, None], 0.5 * F, 0.0)) / rho[:, None]
    assert np.abs(u - uexp).max() < 40 * eps
    # the equilibrium (omega = 1, RR, unforced) against feq - w
    rho0 = np.array([1.03], dt)
    u0 = np.array([[0.05, -0.02, 0.07]], dt)
    feq = feq_shifted(t, rho0, u0, dt)
    eq, _, _ = oracle.q19_collide(feq, np.ones(1, dt), 1.0, np.zeros((1, 6), dt), np.zeros((1, 3), dt))
    assert np.abs(eq - feq).max() < (1e-16 if dt == np.float64 else 1e-7)
    # conservation of the unforced collision
    rng = np.random.default_rng(SEED + 1)
    fs = random_states(t, 64, dt, rng)
    o, _, _ = oracle.q19_collide(fs, np.full(64, 1.7, dt), 0.98, np.zeros((64, 6), dt), np.zeros((64, 3), dt))
    c = np.stack([np.ones(19), t["cx"], t["cy"], t["cz"]]).T
    assert np.abs(o.astype(np.float64) @ c - fs.astype(np.float64) @ c).max() < 40 * eps


def test_positivity_safeguard(q19):
    """States far from equilibrium (noise of half the weights) are blended to the floor (collision.jl:23-40)."""
    oracle, t = q19
    rng = np.random.default_rng(SEED + 2)
    n = 4000
    f = random_states(t, n, np.float64, rng, noise=0.6)
    out, rho, u = oracle.q19_collide(f, np.full(n, 1.9), 1.0, np.zeros((n, 6)), np.zeros((n, 3)))
    plain = out + t["w"][None]
    assert (plain.min(1) > 0).mean() > 0.99   # nearly every cell ends above zero
    # limited cells keep density and momentum (the blend is between states of the same moments)
    c = np.stack([np.ones(19), t["cx"], t["cy"], t["cz"]]).T
    assert np.abs(out @ c - f @ c).max() < 1e-12


def test_periodic_box_generator(q19, oal):
    """Octs of level 1 in Morton order of their origin (generator.jl:280-312), periodic onbr; the
    library's generator (host code) equals the oracle's."""
    oracle, _ = q19
    origin, onbr = oracle.q19_periodic_box(8, 6, 4)
    assert origin.shape == (4 * 3 * 2, 3)

    def spread(v):
        r = 0
        for b in range(21):
            r |= ((v >> b) & 1) << (3 * b)
        return r

    keys = [spread(o[0] // 2 + 1) | spread(o[1] // 2 + 1) << 1 | spread(o[2] // 2 + 1) << 2 for o in origin]
    assert keys == sorted(keys)
    # neighbour of the neighbour in the opposite direction is the oct itself
    for o in range(origin.shape[0]):
        for d in range(27):
            assert onbr[onbr[o, d] - 1, 26 - d] == o + 1
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    n = onbr[o, (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] - 1
                    exp = (origin[o] + 2 * np.array([dx, dy, dz])) % np.array([8, 6, 4])
                    assert (origin[n] == exp).all()
    from openaerolab_alpha_01_b200.octree import PeriodicBox
    b = PeriodicBox(8, 6, 4)
    assert np.array_equal(b.origin, origin) and np.array_equal(b.onbr, onbr)


def _params(nu=0.01, sgs=0, sigma=1.0, F=(0.0, 0.0, 0.0)):
    from openaerolab_alpha_01_b200 import _capi as capi
    p = capi.Q19Params()
    p.abi_version = 1
    p.nu, p.sgs, p.c_wale, p.c_smagorinsky, p.hrr_sigma = nu, sgs, 0.5, 0.1, sigma
    for a in range(3):
        p.body_force[a] = F[a]
    return p


def _fields(origin, n, init, dt, h=0.5):
    """(rho, u, du) of `init` at the slot centres as state.jl:267-305 forms them (dx = 1)."""
    k = np.arange(8)
    cells = origin[:, :, None] + np.stack([k & 1, (k >> 1) & 1, (k >> 2) & 1])[None]
    x, y, z = cells[:, 0] + 0.5, cells[:, 1] + 0.5, cells[:, 2] + 0.5
    rho, ux, uy, uz = (np.broadcast_to(np.asarray(v, np.float64), x.shape) for v in init(x, y, z))
    du = np.zeros((origin.shape[0], 9, 8))
    for a in range(3):
        e = [0.0, 0.0, 0.0]
        e[a] = h
        up, um = init(x + e[0], y + e[1], z + e[2]), init(x - e[0], y - e[1], z - e[2])
        for b in range(3):
            du[:, 3 * a + b] = np.asarray(up[b + 1]) - np.asarray(um[b + 1])
    return rho.astype(dt), np.stack([ux, uy, uz], 1).astype(dt), du.astype(dt)


def test_g03_rest_state(q19):
    """q19_octree_step.jl:30-41: a fluid at rest stays exactly at rest; the mass is exactly n^3."""
    oracle, _ = q19
    origin, onbr = oracle.q19_periodic_box(16, 16, 16)
    L = oracle.OracleQ19Level(onbr, np.float32)
    p = _params()
    rho, u, du = _fields(origin, 16, lambda x, y, z: (1.0, 0.0 * x, 0.0 * x, 0.0 * x), np.float32)
    L.initialise(p, rho, u, du)
    L.step(p, 50)
    assert (L.f == 0).all() and (L.u == 0).all()
    assert L.totals()[0] == 16 ** 3


def g04_init(n):
    s, c, tp = np.sin, np.cos, 2 * np.pi
    return lambda x, y, z: (1.0 + 0.01 * s(tp * x / n) * c(tp * z / n), 0.03 * s(tp * y / n),
                            0.02 * c(tp * z / n), 0.01 * s(tp * x / n))


@pytest.mark.parametrize("dt,tol", [(np.float32, 2e-6), (np.float64, 1e-12)])
@pytest.mark.parametrize("sigma", [1.0, 0.98])
def test_g04_conservation(q19, dt, tol, sigma):
    """q19_octree_step.jl:43-54: mass and momentum over 100 steps, RR and HRR."""
    oracle, _ = q19
    origin, onbr = oracle.q19_periodic_box(16, 16, 16)
    L = oracle.OracleQ19Level(onbr, dt)
    p = _params(sigma=sigma)
    L.initialise(p, *_fields(origin, 16, g04_init(16), dt))
    t0 = L.totals()
    L.step(p, 100)
    t1 = L.totals()
    assert abs(t1[0] - t0[0]) / t0[0] < tol
    assert np.abs(t1[1:4] - t0[1:4]).max() / (16 ** 3 * 0.03) < tol
    assert np.isfinite(L.f).all()


def test_planted_mistake_is_caught(q19):
    """A wrong viscosity in the oracle (a planted mistake) changes the state: the bitwise
    comparisons of the GPU tests are sensitive to one-ulp parameter changes."""
    oracle, _ = q19
    origin, onbr = oracle.q19_periodic_box(8, 8, 8)
    rho, u, du = _fields(origin, 8, g04_init(8), np.float32)
    out = []
    for nu in (0.01, float(np.nextafter(np.float32(0.01), np.float32(1)))):
        L = oracle.OracleQ19Level(onbr, np.float32)
        p = _params(nu=nu, sgs=1, sigma=0.98)
        L.initialise(p, rho, u, du)
        L.step(p, 3)
        out.append(L.f.copy())
    assert not np.array_equal(out[0], out[1])
