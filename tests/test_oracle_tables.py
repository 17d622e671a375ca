"""Oracle D3Q27 tables against the reference's definition (src/collision/lattice.jl:10-60,
src/collision/timestep.jl:2005-2023) and the lattice identities the reference's lattice test
checks for its other velocity sets (tools/tests/q19_octree_lattice.jl:22-79)."""
import itertools

import numpy as np


def test_ordering_is_z_outer_x_inner(oracle_lib):
    t = oracle_lib.d3q27_tables()
    # for z in -1:1, y in -1:1, x in -1:1  ->  k = (cx+1) + 3(cy+1) + 9(cz+1)
    expect = [(x, y, z) for z in (-1, 0, 1) for y in (-1, 0, 1) for x in (-1, 0, 1)]
    got = list(zip(t["cx"].tolist(), t["cy"].tolist(), t["cz"].tolist()))
    assert got == expect
    for k, (x, y, z) in enumerate(expect):
        assert k == (x + 1) + 3 * (y + 1) + 9 * (z + 1)


def test_weights_and_maps(oracle_lib):
    t = oracle_lib.d3q27_tables()
    c = np.stack([t["cx"], t["cy"], t["cz"]], 1)
    d2 = (c ** 2).sum(1)
    w = t["w"]
    assert np.array_equal(w[d2 == 0], [8 / 27])
    assert np.allclose(w[d2 == 1], 2 / 27) and np.allclose(w[d2 == 2], 1 / 54) and np.allclose(w[d2 == 3], 1 / 216)
    assert abs(w.sum() - 1) < 1e-15
    for k in range(27):
        assert np.array_equal(c[t["opp"][k]], -c[k])
        assert np.array_equal(c[t["mirror_y"][k]], c[k] * [1, -1, 1])
        assert np.array_equal(c[t["mirror_z"][k]], c[k] * [1, 1, -1])
        assert t["opp"][k] == 26 - k


def test_isotropy(oracle_lib):
    t = oracle_lib.d3q27_tables()
    c = np.stack([t["cx"], t["cy"], t["cz"]], 1).astype(float)
    w = t["w"]
    for a in range(3):
        assert abs((w * c[:, a]).sum()) < 1e-15
    for a, b in itertools.product(range(3), repeat=2):
        assert abs((w * c[:, a] * c[:, b]).sum() - (a == b) / 3) < 1e-15
    for a, b, cc, d in itertools.product(range(3), repeat=4):
        m4 = (w * c[:, a] * c[:, b] * c[:, cc] * c[:, d]).sum()
        iso = ((a == b) * (cc == d) + (a == cc) * (b == d) + (a == d) * (b == cc)) / 9
        assert abs(m4 - iso) < 1e-15
