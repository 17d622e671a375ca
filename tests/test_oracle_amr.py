"""Block AMR of the D3Q27 path: the oracle's recursion (CPU, no GPU).

The reference has no test of its block-AMR coupling; the gates here are the octree solver's level
gates restated for block levels (tools/tests/q19_octree_levels.jl:70-215): a uniform flow crosses
the refinement interfaces unchanged (G2.0), mass drifts by less than 1e-4 relative over the run
(G2.x conservation), and a smooth wave through a refined patch stays close to the single-level
solution.
"""
import numpy as np
import pytest


def hierarchy(oracle_lib, n_levels=2, bdims=(4, 2, 2), box=None, periodic=(True, True, True)):
    from openaerolab_alpha_01_b200 import amr, solver
    doms = [solver.build_box(*bdims, periodic=periodic)]
    for l in range(1, n_levels):
        parent = doms[-1]
        if box is None:
            # nested slabs around the middle of the domain along x: half the domain for level 1,
            # a quarter for level 2; everything along y and z
            nx = parent.shape[0]
            half = 0.25 / 2 ** (l - 1)
            lo, hi = (nx * (0.5 - half), 0, 0), (nx * (0.5 + half), parent.shape[1], parent.shape[2])
        else:
            lo, hi = [v * 2 ** (l - 1) for v in box[0]], [v * 2 ** (l - 1) for v in box[1]]
        doms.append(amr.refine(parent, amr.blocks_in_box(parent, lo, hi)))
    return doms


def params(taus, **kw):
    from openaerolab_alpha_01_b200 import solver
    return [solver.default_step_params(tau=float(t), **kw) for t in taus]


def init_all(ora, doms, rho_fn, vel_fn):
    for l, d in enumerate(doms):
        gx, gy, gz = d.cell_positions()
        s = 2.0 ** l
        X, Y, Z = (gx - 0.5) / s, (gy - 0.5) / s, (gz - 0.5) / s  # coarse-cell units
        ora.init_equilibrium(l, rho_fn(X, Y, Z), vel_fn(X, Y, Z))


def test_refine_structure(oracle_lib):
    from openaerolab_alpha_01_b200 import amr
    doms = hierarchy(oracle_lib, 3)
    assert [d.n_blocks for d in doms] == [16, 64, 256]
    for parent, child in zip(doms, doms[1:]):
        assert (child.bx_max, child.by_max, child.bz_max) == (2 * parent.bx_max, 2 * parent.by_max, 2 * parent.bz_max)
        pset = {tuple(c) for c in parent.coords.tolist()}
        for c in child.coords.tolist():
            assert ((c[0] + 1) // 2, (c[1] + 1) // 2, (c[2] + 1) // 2) in pset
        # neighbours inside the child level are mutual
        n = child.n_blocks
        for b in range(n):
            for d in range(27):
                v = child.neighbor_table[d, b]
                if v:
                    assert child.neighbor_table[26 - d, v - 1] == b + 1
    assert amr.level_taus(0.55, 3) == pytest.approx([0.7, 0.6, 0.55])


@pytest.mark.parametrize("n_levels", [2, 3])
def test_uniform_flow_crosses_interfaces(oracle_lib, n_levels):
    """G2.0: a uniform flow stays uniform through the refinement interfaces (FP64)."""
    from openaerolab_alpha_01_b200 import amr
    doms = hierarchy(oracle_lib, n_levels)
    ora = oracle_lib.OracleAMR(doms, np.float64)
    u = 0.05
    init_all(ora, doms, lambda X, Y, Z: np.ones_like(X), lambda X, Y, Z: np.stack([u + 0 * X, 0 * X, 0 * X]))
    P = params(amr.level_taus(0.55, n_levels), c_wale=0.0, u_inlet=u)
    ora.advance(P, 4)
    for l in range(n_levels):
        f, rho, vel = ora.state(l)
        assert np.max(np.abs(rho - 1.0)) < 1e-12, l
        assert np.max(np.abs(vel[0] - u)) < 1e-12 and np.max(np.abs(vel[1:])) < 1e-12, l


def wave_setup(oracle_lib, fine_blocks):
    from openaerolab_alpha_01_b200 import amr, solver
    coarse = solver.build_box(4, 4, 1, periodic=(True, True, True))
    blocks = list(range(coarse.n_blocks)) if fine_blocks == "all" else amr.blocks_in_box(coarse, (8, 0, 0), (24, 32, 8))
    return [coarse, amr.refine(coarse, blocks)]


def test_mass_drift_and_smooth_wave(oracle_lib):
    """A shear wave u_x = U sin(k y) (32 coarse cells per wavelength) across a refined slab, with the
    reference's "physical" level-viscosity rule (level_visc_physical = 1: tau_f - 1/2 =
    2 (tau_c - 1/2), uniform physical viscosity, transfer factors tau_f/(2 tau_c) and 2 tau_c/tau_f).
    A hierarchy whose fine level covers the whole domain (restriction and recursion only) matches
    the single-level solution within 0.2 % of U; with the slab (parent interpolation at two
    interfaces) the coarse velocity stays within 3 % of U of it after 40 coarse steps (measured
    2.4 %: the interface error of the scheme, whose density seam the reference documents as
    O(1e-4)), and coarse-level mass drifts by < 1e-4 relative (the coupling is not conservative)."""
    U = 0.02
    k = 2 * np.pi / 32
    rho_fn = lambda X, Y, Z: np.ones_like(X)
    vel_fn = lambda X, Y, Z: np.stack([U * np.sin(k * Y), 0 * X, 0 * X])
    taus = [0.56, 0.62]

    def run(doms, n=40):
        o = oracle_lib.OracleAMR(doms, np.float64)
        init_all(o, doms, rho_fn, vel_fn)
        m0 = o.state(0)[1].sum()
        o.advance(params(taus[:len(doms)], c_wale=0.0, level_visc_physical=1), n)
        return o, m0

    ref, _ = run(wave_setup(oracle_lib, "all")[:1])
    full, _ = run(wave_setup(oracle_lib, "all"))
    slab, m0 = run(wave_setup(oracle_lib, "slab"))
    vr = ref.state(0)[2][0]
    assert np.max(np.abs(full.state(0)[2][0] - vr)) < 0.002 * U
    assert np.max(np.abs(slab.state(0)[2][0] - vr)) < 0.03 * U
    assert abs(slab.state(0)[1].sum() - m0) / m0 < 1e-4
    assert np.all(np.isfinite(slab.state(1)[0]))
