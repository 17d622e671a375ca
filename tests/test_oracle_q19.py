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
import math

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


def _params(nu=0.01, sgs=0, sigma=1.0, F=(0.0, 0.0, 0.0), u_inlet=(0.08, 0.0, 0.0)):
    from openaerolab_alpha_01_b200 import _capi as capi
    p = capi.Q19Params()
    p.abi_version = 1
    p.nu, p.sgs, p.c_wale, p.c_smagorinsky, p.hrr_sigma = nu, sgs, 0.5, 0.1, sigma
    for a in range(3):
        p.body_force[a] = F[a]
        p.u_inlet[a] = u_inlet[a]
    p.force_scale = 1.0
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


# ---- one level with domain faces and a body (generator.jl, stream.jl:205-257) ---------------------

def channel(n, H, angle_deg, seed):
    """The tilted Poiseuille channel of tools/tests/q19_octree_poiseuille.jl:24-50: two slabs
    (closed boxes reaching far beyond the domain) tilted about x, a random sub-cell centre drawn
    from `seed`; periodic in x, slip at the y and z faces. Returns (mesh, centre, unit normal)."""
    import math
    from openaerolab_alpha_01_b200 import octree
    rng = np.random.default_rng(seed)
    a = math.radians(angle_deg)
    Lx, Ly, Lz = 2 * (n // 4), 2 * n, 2 * n
    c = np.array([0.0, Ly / 2 + (rng.random() - 0.5), Lz / 2 + (rng.random() - 0.5)])
    thick, Wh = 4.0 * n, 4 * n

    def rot(p):
        return np.stack([p[..., 0], math.cos(a) * p[..., 1] - math.sin(a) * p[..., 2],
                         math.sin(a) * p[..., 1] + math.cos(a) * p[..., 2]], -1)

    tris = []
    for sign in (1, -1):
        lo = (-Lx, -Wh, H if sign > 0 else -H - thick)
        hi = (2 * Lx, Wh, H + thick if sign > 0 else -H)
        tris.append(rot(octree.box_triangles(lo, hi)) + c)
    spec = octree.MeshSpec(domain=(Lx, Ly, Lz), periodic=(True, False, False),
                           faces=("periodic", "periodic", "slip", "slip", "slip", "slip"))
    return octree.generate(np.concatenate(tris), spec).levels[0], c, np.array([0.0, -math.sin(a), math.cos(a)])


def obstacle_box_mesh():
    """A closed box in a non-periodic domain whose six faces carry six different conditions."""
    from openaerolab_alpha_01_b200 import octree
    tri = octree.box_triangles((5.3, 4.6, 3.7), (9.1, 7.4, 8.2))
    spec = octree.MeshSpec(domain=(16.0, 12.0, 12.0), faces=("inlet", "outlet", "noslip", "freestream",
                                                               "symmetry", "ground"))
    return octree.generate(tri, spec).levels[0]


def mesh_invariants(m):
    """The single-level parts of q19_octree_generator.jl:9-60."""
    no = m.nocts
    on = m.onbr
    assert ((on >= 0) & (on <= no)).all()
    for d in range(27):
        dx, dy, dz = d % 3 - 1, (d // 3) % 3 - 1, d // 9 - 1
        inv = (-dx + 1) + 3 * (-dy + 1) + 9 * (-dz + 1)
        has = on[:, d] > 0
        assert (on[on[has, d] - 1, inv] == np.nonzero(has)[0] + 1).all()
    fluid_octs = (m.kind == 1).any(1)
    assert (on[fluid_octs] > 0).all()
    assert (m.origin % 2 == 0).all() and len({tuple(o) for o in m.origin}) == no
    for ci, s in enumerate(m.cut_slot):
        k, o = (s - 1) % 8, (s - 1) // 8
        assert m.kind[o, k] == 1 and m.cutidx[o, k] == ci + 1
    assert ((m.cut_dir >= 2) & (m.cut_dir <= 19)).all() and ((m.cut_q > 0) & (m.cut_q <= 1)).all()
    assert np.diff(m.cut_off).min() >= 1 and m.cut_off[0] == 1 and m.cut_off[-1] == len(m.cut_dir) + 1
    # special masks: only fluid slots of real octs, never the rest direction
    assert (m.special[m.kind != 1] == 0).all() and (m.special & 1 == 0).all()


@pytest.mark.parametrize("angle", [0.0, 30.0])
def test_generator_channel(oal, angle):
    m, c, nrm = channel(18, 3.0, angle, int(angle) + 18)
    mesh_invariants(m)
    assert m.counts["leak_cells"] == 0 and m.counts["solid"] > 0
    if angle == 0.0:
        # the fluid is exactly the channel: 2H = 6 cells across, the whole periodic length and width
        assert m.counts["fluid_total"] == 8 * 36 * 6
    # fluid slots lie between the plates, solid ones outside
    p = m.slot_centres()
    d = ((p - c[None, :, None]) * nrm[None, :, None]).sum(1)
    assert (np.abs(d[m.kind == 1]) < 3.0).all()
    assert (np.abs(d[m.kind == 2]) > 3.0 - 1e-9).all()


def test_generator_obstacle_box(oal):
    m = obstacle_box_mesh()
    mesh_invariants(m)
    assert m.counts["leak_cells"] == 0
    # the box's cells (centres inside) are solid, everything else of the domain is fluid
    p = m.slot_centres()
    inside = ((p[:, 0] > 5.3) & (p[:, 0] < 9.1) & (p[:, 1] > 4.6) & (p[:, 1] < 7.4) & (p[:, 2] > 3.7) & (p[:, 2] < 8.2))
    real = m.real.astype(bool)[:, None] & np.ones(8, bool)
    assert (m.kind[inside & real] == 2).all()
    assert (m.kind[~inside & real] == 1).all()
    assert m.counts["fluid_total"] + m.counts["solid"] == 16 * 12 * 12


def poiseuille(make_level, n, angle, nu=0.1, Fx=1e-5, steps=None):
    """Run the body-force channel to a steady state; returns (profile error, wall error, friction error).

    The sub-cell offset of the channel is drawn once per angle (seed = angle) and shared by the three
    sizes. The reference draws a new offset per size from Julia's generator (seed angle + n), whose
    values cannot be reproduced here; with a different offset per size the convergence order mixes
    the offsets' effect on the O(1/H^2) wall term (the two walls' Bouzidi q differ by the offset)
    into the ratio of the errors, so a shared offset is what measures the order itself."""
    H = n / 6
    m, c, nrm = channel(n, H, angle, int(angle))
    steps = steps or int(round(5 * H * H / nu))
    u, forces = make_level(m, nu, Fx, steps)
    p = m.slot_centres()
    Ly = 2 * n
    sel = (m.kind == 1) & (np.abs(p[:, 1] - Ly / 2) < Ly / 8)
    d = ((p[:, 1] - c[1]) * nrm[1] + (p[:, 2] - c[2]) * nrm[2])[sel]
    ux = u[:, 0][sel].astype(np.float64)
    A = np.stack([np.ones_like(d), d * d], 1)
    coef = np.linalg.lstsq(A, ux, rcond=None)[0]
    H_eff = math.sqrt(-coef[0] / coef[1])
    umax = Fx * H * H / (2 * nu)
    prof = np.abs(ux - Fx / (2 * nu) * (H * H - d * d)).max() / umax
    body = Fx * m.counts["fluid_total"]
    return prof, H_eff - H, abs(abs(forces[0]) - body) / body


def test_poiseuille_channel_oracle(oal, oracle_lib):
    """q19_octree_poiseuille.jl:77-100 at the smallest size on the oracle: the profile within 20 %."""
    def run(m, nu, Fx, steps):
        from openaerolab_alpha_01_b200 import octree
        d = m.desc()
        L = oracle_lib.OracleQ19Level(m.onbr, np.float64, desc=d)
        p = _params(nu=nu, F=(Fx, 0.0, 0.0))
        rho = np.ones((m.nocts, 8))
        L.initialise(p, rho, np.zeros((m.nocts, 3, 8)), np.zeros((m.nocts, 9, 8)))
        L.step(p, steps, collect=True)
        return L.u, L.forces
    for angle in (0.0, 30.0):
        prof, wall, fric = poiseuille(run, 18, angle)
        assert prof < 0.2, (angle, prof, wall, fric)
