"""Refined octree meshes on the CPU: the generator's invariants and the oracle's coupling gates.

Restated from the reference's tests:
  tools/tests/q19_octree_generator.jl:9-89  invariants of a refined mesh (neighbour symmetry, complete
                                            neighbours of fluid octs, children of covered slots,
                                            ghost donor weights, restriction sources)
  tools/tests/q19_octree_levels.jl:16-23, 70-88   G2.0 uniform flow through a refined box, exact
  tools/tests/q19_octree_levels.jl:177-190        G2.5 mass drift of a periodic box with a refined region
"""
import numpy as np
import pytest

K_FLUID, K_SOLID, K_COVERED, K_GHOST, K_BOUNDARY = 1, 2, 3, 4, 5


def refined_box(n, levels, region_fraction=0.5):
    """Periodic box of n^3 finest cells with a central box refined to the finest level
    (q19_octree_levels.jl:16-23)."""
    from openaerolab_alpha_01_b200 import octree
    L = float(n)
    regions = () if levels == 1 else (octree.Region("box", levels, lo=(L * (0.5 - region_fraction / 2),) * 3,
                                                    hi=(L * (0.5 + region_fraction / 2),) * 3),)
    spec = octree.MeshSpec(domain=(L, L, L), periodic=(True, True, True), levels=levels, dx_finest=1.0, band_fine=4,
                           band=3, regions=regions, faces=("periodic",) * 6)
    return octree.generate(np.zeros((0, 3, 3)), spec)


def refined_slab(n, levels):
    """Periodic box with the slab n/4 <= z < 3n/4 refined (q19_octree_levels.jl:26-33)."""
    from openaerolab_alpha_01_b200 import octree
    L = float(n)
    regions = () if levels == 1 else (octree.Region("box", levels, lo=(0.0, 0.0, L / 4), hi=(L, L, 3 * L / 4)),)
    spec = octree.MeshSpec(domain=(L, L, L), periodic=(True, True, True), levels=levels, dx_finest=1.0, band_fine=4,
                           band=3, regions=regions, faces=("periodic",) * 6)
    return octree.generate(np.zeros((0, 3, 3)), spec)


def refined_invariants(m):
    L = m.nlevels
    for l, lv in enumerate(m.levels, start=1):
        on = lv.onbr
        for d in range(27):
            dx, dy, dz = d % 3 - 1, (d // 3) % 3 - 1, d // 9 - 1
            inv = (-dx + 1) + 3 * (-dy + 1) + 9 * (-dz + 1)
            has = on[:, d] > 0
            assert (on[on[has, d] - 1, inv] == np.nonzero(has)[0] + 1).all()
        assert (on[(lv.kind == K_FLUID).any(1)] > 0).all()
        assert (lv.origin % 2 == 0).all()
        idx = lv.oct_index()
        if l < L:
            fine = m.levels[l]
            fidx = fine.oct_index()
            for o in range(lv.nocts):
                for k in range(8):
                    c = lv.origin[o] + np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
                    child = fidx.get(tuple(2 * c))
                    if lv.kind[o, k] == K_COVERED:
                        assert child is not None and not np.isin(fine.kind[child], (K_GHOST, K_BOUNDARY)).any()
                    elif lv.kind[o, k] in (K_FLUID, K_SOLID):
                        assert child is None or np.isin(fine.kind[child], (K_GHOST, K_SOLID)).all()
        if l > 1:
            coarse = m.levels[l - 2]
            restricted = set(int(s) for s in coarse.restrict_slot)
            for g in range(lv.ghost_slot.shape[0]):
                s = lv.ghost_slot[g] - 1
                assert lv.kind[s // 8, s % 8] == K_GHOST
                assert abs(lv.ghost_w[g].sum() - 1) < 1e-5
                don = lv.ghost_donor[g]
                if not (don != 0).all():
                    inner = [(1 + (m_ & 1)) + 4 * (1 + ((m_ >> 1) & 1)) + 16 * (1 + ((m_ >> 2) & 1)) for m_ in range(8)]
                    outer = np.setdiff1d(np.arange(64), inner)
                    assert (don[outer] == 0).all()
                for d_ in don[don != 0]:
                    kd = coarse.kind[(d_ - 1) // 8, (d_ - 1) % 8]
                    assert kd in (K_FLUID, K_COVERED, K_GHOST)
                    if kd == K_COVERED:
                        assert int(d_) in restricted
        if l < L:
            fine = m.levels[l]
            rf = set(int(s) for s in fine.restrict_slot)
            for r in range(lv.restrict_slot.shape[0]):
                s = lv.restrict_slot[r] - 1
                assert lv.kind[s // 8, s % 8] == K_COVERED
                src = lv.restrict_src[r]
                if lv.restrict_cubic[r]:
                    assert (src != 0).all()
                for c_ in src[src != 0]:
                    kc = fine.kind[(c_ - 1) // 8, (c_ - 1) % 8]
                    assert kc in (K_FLUID, K_GHOST, K_COVERED)
                    if kc == K_COVERED:
                        assert int(c_) in rf


@pytest.mark.parametrize("make", [lambda: refined_box(32, 3), lambda: refined_slab(32, 2)])
def test_refined_generator_invariants(oal, make):
    m = make()
    refined_invariants(m)
    # the leaves partition the domain
    L = m.nlevels
    vol = sum(lv.counts["fluid_total"] * 8.0 ** (L - lv.level) for lv in m.levels)
    assert vol == 32 ** 3
    for lv in m.levels[1:]:
        assert lv.ghost_slot.shape[0] > 0


def oracle_octree(oracle_lib, m, dt, nu=0.005, sgs="none", sigma=1.0, body_force=(0.0, 0.0, 0.0)):
    from openaerolab_alpha_01_b200 import octree
    cfg = octree.test_case_config(m.levels[-1], nu_lattice=nu, precision=dt, sgs=sgs, hrr_sigma=sigma,
                                  body_force=body_force)
    L = m.nlevels
    params = [cfg.params(l, L) for l in range(1, L + 1)]
    descs = [lv.desc() for lv in m.levels]
    T = oracle_lib.OracleQ19Octree(descs, [lv.onbr for lv in m.levels], dt)
    T._keep = (m, descs)
    return T, params, cfg


def level_fields(m, init, dt, nonequilibrium=True):
    """Per level (rho, u, du) of `init` at the slot centres (state.jl:267-305), du over one cell."""
    out = []
    for lv in m.levels:
        p = lv.slot_centres()
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        rho, ux, uy, uz = (np.broadcast_to(np.asarray(v, np.float64), x.shape) for v in init(x, y, z))
        du = None
        if nonequilibrium:
            h = lv.dx / 2
            du = np.zeros((lv.nocts, 9, 8))
            for a in range(3):
                e = [0.0, 0.0, 0.0]
                e[a] = h
                up, um = init(x + e[0], y + e[1], z + e[2]), init(x - e[0], y - e[1], z - e[2])
                for b in range(3):
                    du[:, 3 * a + b] = np.asarray(up[b + 1]) - np.asarray(um[b + 1])
            du = du.astype(dt)
        out.append((rho.astype(dt), np.stack([ux, uy, uz], 1).astype(dt), du))
    return out


def test_g20_uniform_flow_oracle(oracle_lib):
    """G2.0: a uniform stream crosses the interfaces of a 3-level refined box unchanged (< 1e-9)."""
    m = refined_box(32, 3)
    T, params, _ = oracle_octree(oracle_lib, m, np.float64, nu=0.005)
    U0 = 0.04
    T.initialise(params, level_fields(m, lambda x, y, z: (1.0, U0 + 0 * x, 0 * x, 0 * x), np.float64))
    T.advance(params, 64)
    worst = worst_rho = 0.0
    for S, lv in zip(T.levels, m.levels):
        fl = lv.kind == K_FLUID
        u = S.u.transpose(0, 2, 1)[fl]
        worst = max(worst, np.abs(u[:, 0] - U0).max(), np.abs(u[:, 1:]).max())
        worst_rho = max(worst_rho, np.abs(S.rho[fl] - 1).max())
    assert worst < 1e-9 and worst_rho < 1e-9


def g25_init(n):
    s, c, tp = np.sin, np.cos, 2 * np.pi
    return lambda x, y, z: (1.0 + 0.01 * s(tp * x / n) * c(tp * z / n), 0.03 * s(tp * y / n),
                            0.02 * c(tp * z / n) * s(tp * x / n), 0.01 * s(tp * x / n))


def test_g25_mass_drift_oracle(oracle_lib):
    """G2.5 (shortened to 2 n coarse steps on the CPU): the mass of a periodic box with a 3-level
    refined region drifts by less than 1e-4."""
    n = 32
    m = refined_box(n, 3)
    T, params, _ = oracle_octree(oracle_lib, m, np.float64, nu=0.01)
    T.initialise(params, level_fields(m, g25_init(n), np.float64))
    m0 = T.totals()[0]
    T.advance(params, 2 * n)
    assert np.isfinite(T.levels[-1].f).all()
    assert abs(T.totals()[0] - m0) / m0 < 1e-4
