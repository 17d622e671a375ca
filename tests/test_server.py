"""Serving: request generation (CPU) and continuous batching (GPU): every served result equals the
same request solved alone, while requests join and leave the resident mix — D3Q27 solves in the
shared block pool and D3Q39 KBC solves as levels on their own streams beside it."""
import math

import numpy as np
import pytest

from openaerolab_alpha_01_b200 import server


def test_request_stream_is_seeded_and_in_range():
    a = server.make_requests(200, rate=20.0, steps=100, seed=3)
    b = server.make_requests(200, rate=20.0, steps=100, seed=3)
    assert [(r.arrival, r.n, r.kind, r.re) for r in a] == [(r.arrival, r.n, r.kind, r.re) for r in b]
    assert all(32 <= r.n <= 192 and r.n % 8 == 0 for r in a)
    assert all(100 <= r.re <= 5000 for r in a)
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 1 / 20.0) < 0.02          # Poisson rate
    assert 0.3 < np.mean([r.kind == "channel" for r in a]) < 0.7


def test_request_mix_with_kbc_share():
    a = server.make_requests(400, rate=20.0, steps=100, seed=4, kbc_share=0.5)
    kbc = [r for r in a if r.operator == "entropic"]
    assert 0.4 < len(kbc) / len(a) < 0.6
    assert 0.3 < np.mean([r.kind == "channel" for r in kbc]) < 0.7
    assert all(r.operator == "cumulant" for r in server.make_requests(50, seed=4))


def test_pool_block_costs():
    rb, gb = server.block_bytes("f16")
    assert rb > gb > 27 * 512 * 2


@pytest.mark.gpu
def test_served_results_equal_solving_alone(oal):
    reqs = server.make_requests(8, rate=200.0, steps=40, n_min=16, n_max=24, seed=11)
    served, states = server.serve(reqs, budget_bytes=30e6, storage="f32", tick_steps=15, keep_states=True)
    assert served["completed"] == 8
    assert all(r.done > r.admitted >= r.arrival for r in reqs)
    reqs2 = server.make_requests(8, rate=200.0, steps=40, n_min=16, n_max=24, seed=11)
    seq, alone = server.serve_sequential(reqs2, storage="f32", keep_states=True)
    for r in reqs:
        assert np.array_equal(states[r.rid], alone[r.rid]), r.rid
    # the small budget forced queueing: not everything was admitted at its arrival
    assert any(r.admitted - r.arrival > 1e-3 for r in reqs)


@pytest.mark.gpu
def test_request_larger_than_the_pool_is_rejected(oal):
    reqs = server.make_requests(2, rate=200.0, steps=10, n_min=32, n_max=32, seed=2)
    served, _ = server.serve(reqs, budget_bytes=2e6, storage="f32", tick_steps=5)
    assert served["rejected"] == 2 and served["completed"] == 0


@pytest.mark.gpu
def test_served_mix_with_kbc_equals_solving_alone(oal):
    """D3Q39 and D3Q27 requests served together: each result is bit-identical to the request run
    alone, and the KBC share of the budget forces some KBC requests to wait for a slot."""
    kw = dict(rate=200.0, steps=30, n_min=16, n_max=24, seed=7, kbc_share=0.5)
    reqs = server.make_requests(10, **kw)
    assert any(r.operator == "entropic" for r in reqs) and any(r.operator == "cumulant" for r in reqs)
    budget = 40e6
    served, states = server.serve(reqs, budget_bytes=budget, storage="f32", tick_steps=10, keep_states=True,
                                  kbc_budget_share=24 ** 3 * server.KBC_BYTES_PER_CELL * 1.5 / budget)
    assert served["completed"] == 10 and served["completed_d3q39"] == sum(r.operator == "entropic" for r in reqs)
    reqs2 = server.make_requests(10, **kw)
    seq, alone = server.serve_sequential(reqs2, storage="f32", keep_states=True)
    seq_cs = {r.rid: r.checksum for r in reqs2}
    for r in reqs:
        assert np.array_equal(states[r.rid], alone[r.rid]), (r.rid, r.operator)
        assert all(np.isfinite(r.checksum)) and r.checksum == seq_cs[r.rid]
        if r.operator == "entropic" and r.kind == "channel":
            # the surface-stress drag on the sphere: in the stream direction
            assert r.drag > 0, r.checksum
    kbc = [r for r in reqs if r.operator == "entropic"]
    assert len(kbc) < 2 or any(r.admitted - r.arrival > 1e-3 for r in kbc)
