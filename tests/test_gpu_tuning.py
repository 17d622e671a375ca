"""Launch tuning and the autotuner (oal_level_autotune, oal_batch_autotune): neither the L2
prefetch distance nor the persistent launch of the x-pair kernel changes a result bit; the
autotuner times every candidate, keeps the fastest and leaves the level or the pool in the state
it found."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200.cases import sphere_channel_case, taylor_green_case
from openaerolab_alpha_01_b200.solver import Batch, Geometry, Level


@pytest.mark.parametrize("storage", ["f16", "bf16", "f32"])
def test_launch_tuning_changes_no_bit(oal, storage):
    case = sphere_channel_case(64, 32, 32, diameter=8.0, centre_x=16.0, u_inlet=0.05, re=200.0)
    g = Geometry(case.dom)
    out = []
    for pf, pers in ((0, False), (148 * 4, False), (148 * 16, False), (0, True), (148 * 4, True)):
        L = Level(g, storage=storage)
        L.prefetch_ctas = pf
        L.persistent = pers
        assert L.prefetch_ctas == pf and L.persistent == pers
        L.init_equilibrium(case.rho, case.vel)
        for _ in range(3):
            L.perform_timestep(case.params)
        L.execute_timestep_batch(case.params, 8)
        out.append((L.state()[0], L.forces()))
        L.close()
    g.close()
    for f, F in out[1:]:
        assert np.array_equal(f, out[0][0]) and np.array_equal(F, out[0][1])


def test_level_autotune_keeps_the_state(oal):
    case = sphere_channel_case(128, 64, 64, diameter=12.0, centre_x=32.0, u_inlet=0.05, re=300.0)
    g = Geometry(case.dom)
    L = Level(g, storage="f16")
    L.init_equilibrium(case.rho, case.vel)
    L.execute_timestep_batch(case.params, 10)
    before = L.state()
    r = L.autotune(case.params, 20)
    after = L.state()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    cands = [(v, q) for v, q, _ in r["candidates"]]
    assert len(cands) == capi.OAL_TUNE_CANDIDATES and cands[0] == (0, 0) and (r["prefetch_ctas"], int(r["persistent"])) in cands
    assert {q for _, q in cands} == {0, 1}
    assert all(t > 0 for _, _, t in r["candidates"])
    best = min(r["candidates"], key=lambda c: c[2])
    assert (r["prefetch_ctas"], int(r["persistent"])) == best[:2]
    # stepping on after tuning equals stepping a level that was never tuned
    M = Level(g, storage="f16")
    M.init_equilibrium(case.rho, case.vel)
    M.execute_timestep_batch(case.params, 16)
    L.execute_timestep_batch(case.params, 6)
    assert np.array_equal(L.state()[0], M.state()[0])
    L.close(); M.close(); g.close()


def test_batch_autotune_keeps_the_members(oal):
    cases = [taylor_green_case(n, u0=0.05, re=400.0) for n in (32, 48, 64)]
    geoms = [Geometry(c.dom) for c in cases]
    B = Batch(storage="f16", max_real_blocks=1024, max_ghost_blocks=1024, max_mask_blocks=16, max_members=4)
    ids = [B.add(g, c.params, c.rho, c.vel) for g, c in zip(geoms, cases)]
    B.advance(4)
    before = [B.state(m)[0] for m in ids]
    r = B.autotune(10)
    assert (r["prefetch_ctas"], int(r["persistent"])) in [(v, q) for v, q, _ in r["candidates"]]
    for m, f in zip(ids, before):
        assert np.array_equal(B.state(m)[0], f)
    B.prefetch_ctas = 0
    B.persistent = False
    B.advance(6)
    ref = [B.state(m)[0] for m in ids]
    B.close()
    # a pool that never prefetches reaches the same populations
    C_ = Batch(storage="f16", max_real_blocks=1024, max_ghost_blocks=1024, max_mask_blocks=16, max_members=4)
    ids2 = [C_.add(g, c.params, c.rho, c.vel) for g, c in zip(geoms, cases)]
    C_.prefetch_ctas = 148 * 8
    C_.persistent = True
    C_.advance(10)
    for m, f in zip(ids2, ref):
        assert np.array_equal(C_.state(m)[0], f)
    C_.close()
    for g in geoms:
        g.close()
