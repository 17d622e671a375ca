"""Batched stepping (oal_batch_*): every member's result is bit-identical to the same case run
alone, across storages, mixed case kinds, membership changes and pool admission."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200.cases import sphere_channel_case, taylor_green_case
from openaerolab_alpha_01_b200.solver import Batch, Geometry, Level


def mixed_cases():
    return [taylor_green_case(16, u0=0.05, re=100.0, c_wale=0.2),
            sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0),
            taylor_green_case(24, u0=0.03, re=400.0, c_wale=0.0, phase=(1.5, 2.5)),
            sphere_channel_case(24, 16, 16, diameter=5.0, centre_x=8.0, u_inlet=0.04, re=80.0,
                                solid_bc=capi.OAL_SOLID_FULLWAY)]


def alone(case, storage, steps):
    g = Geometry(case.dom)
    L = Level(g, storage=storage)
    L.init_equilibrium(case.rho, case.vel)
    L.execute_timestep_batch(case.params, steps)
    f, rho, vel = L.state()
    out = (f, rho, vel, L.forces(), L.mass_momentum())
    L.close(); g.close()
    return out


@pytest.mark.parametrize("storage", ["f16", "f32", "f64"])
def test_members_match_alone_bitwise(oal, storage):
    cases = mixed_cases()
    steps = 9
    B = Batch(storage=storage, max_real_blocks=256, max_ghost_blocks=256, max_mask_blocks=64, max_members=8)
    geoms = [Geometry(c.dom) for c in cases]
    ids = [B.add(g, c.params, c.rho, c.vel) for g, c in zip(geoms, cases)]
    B.advance(4)
    B.advance(5)
    for c, m in zip(cases, ids):
        f, rho, vel, force, mm = alone(c, storage, steps)
        fb, rb, vb = B.state(m)
        assert np.array_equal(fb, f) and np.array_equal(vb, vel) and np.array_equal(rb, rho), c.name
        assert np.array_equal(B.forces(m), force), c.name
        assert np.array_equal(B.mass_momentum(m), mm), c.name
    B.close()


def test_membership_changes_leave_others_untouched(oal):
    cases = mixed_cases()
    B = Batch(storage="f32", max_real_blocks=256, max_ghost_blocks=256, max_mask_blocks=64, max_members=8)
    geoms = [Geometry(c.dom) for c in cases]
    a = B.add(geoms[0], cases[0].params, cases[0].rho, cases[0].vel)
    b = B.add(geoms[1], cases[1].params, cases[1].rho, cases[1].vel)
    B.advance(3)
    c = B.add(geoms[2], cases[2].params, cases[2].rho, cases[2].vel)   # joins mid-run
    B.remove(b)                                                         # leaves mid-run
    d = B.add(geoms[3], cases[3].params, cases[3].rho, cases[3].vel)   # reuses the freed blocks
    B.advance(4)
    fa = alone(cases[0], "f32", 7)[0]
    fc = alone(cases[2], "f32", 4)[0]
    fd = alone(cases[3], "f32", 4)[0]
    assert np.array_equal(B.state(a)[0], fa)
    assert np.array_equal(B.state(c)[0], fc)
    assert np.array_equal(B.state(d)[0], fd)
    assert B.info()["members"] == 3
    B.close()


def test_admission_by_pool_capacity(oal):
    case = taylor_green_case(32)  # 64 blocks
    g = Geometry(case.dom)
    B = Batch(storage="f16", max_real_blocks=130, max_ghost_blocks=0, max_mask_blocks=0, max_members=4)
    assert B.try_add(g, case.params, case.rho, case.vel) is not None
    m2 = B.try_add(g, case.params, case.rho, case.vel)
    assert m2 is not None
    assert B.try_add(g, case.params, case.rho, case.vel) is None   # 3 x 64 > 130
    B.remove(m2)
    assert B.try_add(g, case.params, case.rho, case.vel) is not None
    B.close()


@pytest.mark.parametrize("storage", ["f16", "f32"])
def test_member_with_bouzidi_walls_matches_alone(oal, storage):
    """A member with linear Bouzidi walls (oal_batch_set_bouzidi) beside members without: its
    populations equal the same case stepped alone with oal_level_set_bouzidi, bit for bit."""
    from openaerolab_alpha_01_b200.bouzidi import sphere_qmap
    ch = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0,
                             solid_bc=capi.OAL_SOLID_BOUZIDI)
    ch.params.collect_forces = 0
    cells, q = sphere_qmap(ch.dom, (10.0, 8.0, 8.0), 3.0)
    others = [taylor_green_case(16, u0=0.05, re=100.0, c_wale=0.2),
              sphere_channel_case(24, 16, 16, diameter=5.0, centre_x=8.0, u_inlet=0.04, re=80.0)]
    steps = 8
    g = Geometry(ch.dom)
    L = Level(g, storage=storage)
    L.init_equilibrium(ch.rho, ch.vel)
    L.set_bouzidi(cells, q, ff_fallback=1)
    L.execute_timestep_batch(ch.params, steps)
    ref = L.state()[0]
    L.close()
    geoms = [Geometry(c.dom) for c in others]
    B = Batch(storage=storage, max_real_blocks=256, max_ghost_blocks=256, max_mask_blocks=64, max_members=4)
    ids = [B.add(gg, c.params, c.rho, c.vel) for gg, c in zip(geoms, others)]
    m = B.add(g, ch.params, ch.rho, ch.vel)
    B.set_bouzidi(m, cells, q, ff_fallback=1)
    B.advance(steps)
    assert np.array_equal(B.state(m)[0], ref)
    for i, c in zip(ids, others):
        assert np.array_equal(B.state(i)[0], alone(c, storage, steps)[0])
    B.close()
    for gg in geoms:
        gg.close()
    g.close()


def test_large_channel_member_matches_alone(oal):
    """A channel whose sphere spans more than 128 general-kernel CTAs: the drag summed by the
    level's last CTA and by the pool's per-member reduction take the same order (same bits)."""
    big = sphere_channel_case(128, 64, 64, diameter=24.0, centre_x=32.0, u_inlet=0.05, re=200.0)
    small = taylor_green_case(16, u0=0.05, re=100.0, c_wale=0.2)
    steps = 6
    f, rho, vel, force, mm = alone(big, "f16", steps)
    geoms = [Geometry(c.dom) for c in (small, big)]
    B = Batch(storage="f16", max_real_blocks=1100, max_ghost_blocks=1100, max_mask_blocks=256, max_members=2)
    ids = [B.add(g, c.params, c.rho, c.vel) for g, c in zip(geoms, (small, big))]
    B.advance(steps)
    assert np.array_equal(B.state(ids[1])[0], f)
    assert np.array_equal(B.forces(ids[1]), force)
    assert np.array_equal(B.mass_momentum(ids[1]), mm)
    B.close()
    for g in geoms:
        g.close()


def test_member_of_a_pool_past_2_31_elements_matches_alone(oal):
    """A pool whose population buffer holds more than 2^31 elements (160,000 blocks, the size class
    of the serving pool): the members' raw ghost copies are still a copy list (their element
    indices use all 32 bits), so a channel member stores the bits it stores alone."""
    case = sphere_channel_case(64, 32, 32, diameter=8.0, centre_x=16.0, u_inlet=0.05, re=300.0)
    steps = 120
    f, rho, vel, force, mm = alone(case, "f16", steps)
    g = Geometry(case.dom)
    B = Batch(storage="f16", max_real_blocks=150_000, max_ghost_blocks=10_000, max_mask_blocks=64, max_members=2)
    m = B.add(g, case.params, case.rho, case.vel)
    B.advance(steps)
    assert np.array_equal(B.state(m)[0], f)
    assert np.array_equal(B.forces(m), force) and np.array_equal(B.mass_momentum(m), mm)
    B.close(); g.close()
