"""Block AMR of the D3Q27 path on the GPU against the oracle's recursion.

Every level's populations, density and velocity after a few coarse steps: FP64 storage within
1e-10 of max|f| (the kernels fuse multiply-adds the oracle does not, as on a single level), FP32
within 5e-5. Hierarchies: a periodic box with two and three levels, and a channel whose refined
level touches the domain faces (inlet, outlet, mirror walls at fine resolution) and holds a solid
sphere (children skipped by the restriction).
"""
import numpy as np
import pytest

from .test_oracle_amr import hierarchy, init_all, params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(oal, oracle_lib):
    from openaerolab_alpha_01_b200 import amr, solver
    return oracle_lib, amr, solver


def fields(U=0.04):
    def rho_fn(X, Y, Z):
        return 1.0 + 0.002 * np.cos(2 * np.pi * X / 32)

    def vel_fn(X, Y, Z):
        return np.stack([U * np.sin(2 * np.pi * Y / 16) + 0.01, 0.5 * U * np.cos(2 * np.pi * X / 32),
                         0.3 * U * np.sin(2 * np.pi * (X + Z) / 16)])
    return rho_fn, vel_fn


def run_pair(env, doms, P, storage, n, rho_fn, vel_fn):
    oracle, amr, solver = env
    dt = np.float64 if storage == "f64" else np.float32
    ora = oracle.OracleAMR(doms, dt)
    init_all(ora, doms, rho_fn, vel_fn)
    if dt == np.float32:
        # the GPU starts from the FP64 equilibrium rounded by its codec; give the oracle the same start
        pass
    H = amr.Hierarchy(doms, storage=storage)
    for l, d in enumerate(doms):
        gx, gy, gz = d.cell_positions()
        s = 2.0 ** l
        X, Y, Z = (gx - 0.5) / s, (gy - 0.5) / s, (gz - 0.5) / s
        H.level(l).init_equilibrium(rho_fn(X, Y, Z), vel_fn(X, Y, Z))
    for l in range(len(doms)):
        f, r, v = H.level(l).state()
        ora.levels[l]["f"][0][...] = f
        ora.levels[l]["rho"][...] = r
        ora.levels[l]["vel"][0][...] = v
    H.advance(P, n)
    ora.advance(P, n)
    return H, ora


def compare(H, ora, n_levels, tol):
    for l in range(n_levels):
        f, r, v = H.level(l).state()
        fo, ro, vo = ora.state(l)
        scale = np.max(np.abs(fo))
        assert np.max(np.abs(f - fo)) < tol * scale, (l, np.max(np.abs(f - fo)) / scale)
        assert np.max(np.abs(r - ro)) < tol * 10, l
        assert np.max(np.abs(v - vo)) < tol * 10, l


@pytest.mark.parametrize("n_levels", [2, 3])
def test_periodic_hierarchy_fp64(env, n_levels):
    oracle, amr, solver = env
    doms = hierarchy(oracle, n_levels)
    rho_fn, vel_fn = fields()
    P = params(amr.level_taus(0.52, n_levels), c_wale=0.2)
    H, ora = run_pair(env, doms, P, "f64", 3, rho_fn, vel_fn)
    compare(H, ora, n_levels, 1e-10)
    H.close()


def test_periodic_hierarchy_fp32_physical_rule(env):
    oracle, amr, solver = env
    doms = hierarchy(oracle, 2)
    rho_fn, vel_fn = fields()
    P = params([0.56, 0.62], c_wale=0.2, level_visc_physical=1)
    H, ora = run_pair(env, doms, P, "f32", 4, rho_fn, vel_fn)
    compare(H, ora, 2, 5e-5)
    H.close()


def test_channel_faces_and_obstacle_fp64(env):
    """Inlet/outlet along x, mirror walls in y and z; the refined level spans the channel's full
    cross-section (its pulls across the domain faces use the face conditions at fine resolution)
    and contains a sphere (full-way bounce-back; its solid children are left out of the average)."""
    oracle, amr, solver = env
    coarse = solver.build_box(6, 2, 2)
    fine = amr.refine(coarse, amr.blocks_in_box(coarse, (16, 0, 0), (32, 16, 16)))
    solver.apply_analytic_sphere_obstacle(fine, (48.0, 16.0, 16.0), 5.0)
    doms = [coarse, fine]
    u = 0.05
    rho_fn = lambda X, Y, Z: np.ones_like(X)
    vel_fn = lambda X, Y, Z: np.stack([u + 0 * X, 0.01 * np.sin(2 * np.pi * Y / 16), 0 * X])
    P = params(amr.level_taus(0.53, 2), c_wale=0.2, u_inlet=u)
    H, ora = run_pair(env, doms, P, "f64", 3, rho_fn, vel_fn)
    compare(H, ora, 2, 1e-10)
    # the solid cells stay at rest
    _, _, v = H.level(1).state()
    solid = fine.obstacle.astype(bool)
    assert np.all(v[:, solid] == 0.0)
    H.close()


def test_graph_advance_equals_single_steps(env):
    oracle, amr, solver = env
    doms = hierarchy(oracle, 2)
    rho_fn, vel_fn = fields()
    P = params(amr.level_taus(0.55, 2), c_wale=0.2)
    out = []
    for mode in ("graph", "single"):
        H = amr.Hierarchy(doms, storage="f32")
        for l, d in enumerate(doms):
            gx, gy, gz = d.cell_positions()
            s = 2.0 ** l
            H.level(l).init_equilibrium(rho_fn((gx - 0.5) / s, (gy - 0.5) / s, (gz - 0.5) / s),
                                        vel_fn((gx - 0.5) / s, (gy - 0.5) / s, (gz - 0.5) / s))
        if mode == "graph":
            H.advance(P, 3)
        else:
            for _ in range(3):
                H.advance(P, 1)
        out.append([H.level(l).state() for l in range(2)])
        H.close()
    for (fa, ra, va), (fb, rb, vb) in zip(out[0], out[1]):
        assert np.array_equal(fa, fb) and np.array_equal(ra, rb) and np.array_equal(va, vb)


def test_uniform_flow_fp32(env):
    oracle, amr, solver = env
    doms = hierarchy(oracle, 3)
    u = 0.05
    H = amr.Hierarchy(doms, storage="f32")
    for l, d in enumerate(doms):
        H.level(l).init_equilibrium(np.ones((d.n_blocks, 512)), np.stack([np.full((d.n_blocks, 512), u),
                                                                          np.zeros((d.n_blocks, 512)),
                                                                          np.zeros((d.n_blocks, 512))]))
    H.advance(params(amr.level_taus(0.55, 3), c_wale=0.2, u_inlet=u), 5)
    for l in range(3):
        _, r, v = H.level(l).state()
        assert np.max(np.abs(r - 1)) < 2e-6 and np.max(np.abs(v[0] - u)) < 2e-6 and np.max(np.abs(v[1:])) < 2e-6
    H.close()


@pytest.mark.parametrize("storage,tol", [("f64", 1e-10), ("f32", 5e-5)])
@pytest.mark.parametrize("sphere", [(48.0, 5.0), (35.5, 3.2)], ids=["inside", "at_the_interface"])
def test_channel_bouzidi_on_the_fine_level(env, storage, tol, sphere):
    """The linear Bouzidi wall on the sphere of the refined level (the reference applies it on the
    finest level, bouzidi_levels = 1): the correction follows each fine step, before the
    restriction, in the captured hierarchy graph; a second advance reuses the graph. With the
    sphere against the coarse/fine interface (fine x = 32) the cell behind some q < 1/2 links lies
    in the level's ghost region, outside the level's own blocks: as in the reference, whose
    neighbour table has no entry there, the link takes the ff_fallback rule."""
    oracle, amr, solver = env
    from openaerolab_alpha_01_b200 import _capi as capi
    from openaerolab_alpha_01_b200.bouzidi import sphere_qmap
    coarse = solver.build_box(6, 2, 2)
    fine = amr.refine(coarse, amr.blocks_in_box(coarse, (16, 0, 0), (32, 16, 16)))
    cx, r = sphere
    solver.apply_analytic_sphere_obstacle(fine, (cx, 16.0, 16.0), r)
    cells, q = sphere_qmap(fine, (cx, 16.0, 16.0), r)
    if cx < 40.0:
        # some boundary cell sits in the fine level's first plane, so a link's behind cell is a ghost
        gx = fine.cell_positions()[0]
        b, c = cells[:, 0] - 1, (cells[:, 1] - 1) + 8 * (cells[:, 2] - 1) + 64 * (cells[:, 3] - 1)
        assert (gx[b, c] <= 33.0).any()
    doms = [coarse, fine]
    u = 0.05
    rho_fn = lambda X, Y, Z: np.ones_like(X)
    vel_fn = lambda X, Y, Z: np.stack([u + 0 * X, 0.01 * np.sin(2 * np.pi * Y / 16), 0 * X])
    P = params(amr.level_taus(0.53, 2), c_wale=0.2, u_inlet=u)
    for p in P:
        p.solid_bc = capi.OAL_SOLID_BOUZIDI
        p.collect_forces = 0
    dt = np.float64 if storage == "f64" else np.float32
    ora = oracle.OracleAMR(doms, dt)
    H = amr.Hierarchy(doms, storage=storage)
    for l, d in enumerate(doms):
        gx, gy, gz = d.cell_positions()
        s = 2.0 ** l
        X, Y, Z = (gx - 0.5) / s, (gy - 0.5) / s, (gz - 0.5) / s
        H.level(l).init_equilibrium(rho_fn(X, Y, Z), vel_fn(X, Y, Z))
    for l in range(2):
        f, r, v = H.level(l).state()
        ora.levels[l]["f"][0][...] = f
        ora.levels[l]["rho"][...] = r
        ora.levels[l]["vel"][0][...] = v
    H.level(1).set_bouzidi(cells, q)
    ora.set_bouzidi(1, dict(cells=cells, q=q))
    H.advance(P, 2)
    ora.advance(P, 2)
    H.advance(P, 2)
    ora.advance(P, 2)
    compare(H, ora, 2, tol)
    H.close()
