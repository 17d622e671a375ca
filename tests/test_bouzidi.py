"""Linear Bouzidi wall (bc_scheme "bouzidi_linear", src/geometry/bouzidi_kernel.jl:150-380): the q-map
builder (bouzidi_setup.jl / bouzidi_math.jl, analytic sphere) and the oracle's correction, on the CPU.

The reference ships no fixture for this kernel, so the oracle is pinned on the closed forms the
kernel reduces to: q = 1/2 is half-way bounce-back, q = 1 the mean of f*_k and f*_opp k, and a
missing support cell falls back to f*_k (halfway_bb), w_k rho (wall_eq) or f*_opp k (bounce_back),
each checked against a direct Python evaluation of the formulas on random populations.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from openaerolab_alpha_01_b200.bouzidi import CX, CY, CZ, ray_sphere_first_hit, sphere_qmap
from openaerolab_alpha_01_b200.cases import sphere_channel_case
from openaerolab_alpha_01_b200.solver import apply_analytic_sphere_obstacle, build_box

W = np.array([8 / 27 if d == 0 else 2 / 27 if d == 1 else 1 / 54 if d == 2 else 1 / 216
              for d in (CX ** 2 + CY ** 2 + CZ ** 2)])


def _p(a):
    return None if a is None else a.ctypes.data


def correct(dom, cells, q, fpost, ff=0, rel=0.0, abs_=0.0, q_min=0.001):
    out = fpost.copy()
    qf = np.asarray(q, np.float16).astype(np.float32)
    rc = oracle.lib().ora_bouzidi_linear_f64(dom.n_blocks, _p(np.ascontiguousarray(dom.neighbor_table)),
                                             _p(dom.obstacle), cells.shape[0], _p(np.ascontiguousarray(cells)),
                                             _p(np.ascontiguousarray(qf)), q_min, ff, rel, abs_, _p(fpost), _p(out))
    assert rc == 0
    return out


def wall_box():
    """Two blocks along x; the cells of x-layer 12 (global, 1-based) and beyond are solid."""
    dom = build_box(2, 1, 1)
    gx, _, _ = dom.cell_positions()
    dom.obstacle = (gx >= 12).astype(np.uint8)
    return dom


def test_q_half_is_halfway_bounce_back_and_q_one_the_mean():
    dom = wall_box()
    rng = np.random.default_rng(1)
    fpost = rng.uniform(0.01, 0.1, (27, dom.n_blocks, 512))
    # the fluid cell x = 11 (block 2, local x 3) at y = z = 4 has its +x links into the wall
    cell = np.array([[2, 3, 4, 4]], np.int32)
    ci = 2 + 8 * 3 + 64 * 3
    for qv, expect in ((0.5, lambda k: fpost[k, 1, ci]),
                       (1.0, lambda k: 0.5 * fpost[k, 1, ci] + 0.5 * fpost[26 - k, 1, ci])):
        q = np.zeros((1, 27))
        links = [k for k in range(27) if CX[k] == 1]
        q[0, links] = qv
        out = correct(dom, cell, q, fpost)
        for k in links:
            assert out[26 - k, 1, ci] == pytest.approx(expect(k), rel=1e-14)
        untouched = np.ones(27, bool)
        untouched[[26 - k for k in links]] = False
        assert np.array_equal(out[untouched], fpost[untouched])
        assert np.array_equal(out[:, 0], fpost[:, 0])


@pytest.mark.parametrize("ff", [0, 1, 2])
def test_small_q_with_and_without_support(ff):
    dom = wall_box()
    rng = np.random.default_rng(2)
    fpost = rng.uniform(0.01, 0.1, (27, dom.n_blocks, 512))
    # fluid cell global x = 11: its support x_ff = x - c_k (x = 10) is fluid, then made solid
    k = 14  # c = (+1, 0, 0)
    q = np.zeros((1, 27))
    q[0, k] = 0.3
    cell = np.array([[2, 3, 4, 4]], np.int32)
    ci, cb = 2 + 8 * 3 + 64 * 3, 1 + 8 * 3 + 64 * 3
    c1 = 2.0 * float(np.float16(0.3))  # q is stored as binary16
    out = correct(dom, cell, q, fpost, ff=ff)
    assert out[12, 1, ci] == pytest.approx(c1 * fpost[k, 1, ci] + (1 - c1) * fpost[k, 1, cb], rel=1e-14)
    dom.obstacle = dom.obstacle.copy()
    dom.obstacle[1, cb] = 1
    out = correct(dom, cell, q, fpost, ff=ff)
    fallback = {0: fpost[k, 1, ci], 1: W[k] * fpost[:, 1, ci].sum(), 2: fpost[12, 1, ci]}[ff]
    assert out[12, 1, ci] == pytest.approx(c1 * fpost[k, 1, ci] + (1 - c1) * fallback, rel=1e-14)


def test_support_across_a_block_face_and_the_limiter():
    dom = wall_box()
    rng = np.random.default_rng(3)
    fpost = rng.uniform(0.01, 0.1, (27, dom.n_blocks, 512))
    # fluid cell at local x = 1 of block 2: its support x - c_k lies in block 1 (local x = 8)
    k = 14
    q = np.zeros((1, 27))
    q[0, k] = 0.2
    cell = np.array([[2, 1, 5, 6]], np.int32)
    ci, cb = 0 + 8 * 4 + 64 * 5, 7 + 8 * 4 + 64 * 5
    out = correct(dom, cell, q, fpost)
    c1 = 2.0 * float(np.float16(0.2))
    raw = c1 * fpost[k, 1, ci] + (1 - c1) * fpost[k, 0, cb]
    assert out[12, 1, ci] == pytest.approx(raw, rel=1e-14)
    # limiter: clamp to w_opp rho +- rel_cap |w_opp rho|
    target = W[12] * fpost[:, 1, ci].sum()
    out = correct(dom, cell, q, fpost, rel=1e-3)
    cap = float(np.float32(1e-3)) * target  # the caps are float32 parameters
    assert out[12, 1, ci] == pytest.approx(min(max(raw, target - cap), target + cap), rel=1e-14)
    # q at or below the threshold: nothing changes
    q[0, k] = 0.0005
    assert np.array_equal(correct(dom, cell, q, fpost), fpost)


def test_sphere_qmap_links_and_distances():
    dom = build_box(4, 2, 2)
    centre, radius = (16.0, 8.0, 8.0), 4.3
    apply_analytic_sphere_obstacle(dom, centre, radius)
    cells, q = sphere_qmap(dom, centre, radius)
    assert cells.shape[0] > 0 and q.shape == (cells.shape[0], 27) and q.dtype == np.float16
    solid = dom.obstacle != 0
    coords = dom.coords
    lookup = {tuple(c): i for i, c in enumerate(coords)}
    for (b, x, y, z), qr in zip(cells, q):
        assert not solid[b - 1, (x - 1) + 8 * (y - 1) + 64 * (z - 1)]
        assert (qr > 0).any() and qr[13] == 0
        g = (coords[b - 1] - 1) * 8 + np.array([x, y, z])
        for k in np.nonzero(qr)[0]:
            c = np.array([CX[k], CY[k], CZ[k]])
            n = g + c
            nb = lookup[tuple((n - 1) // 8 + 1)]
            lc = (n - 1) % 8
            assert solid[nb, lc[0] + 8 * lc[1] + 64 * lc[2]]
            # a scalar evaluation of the ray-sphere distance (bouzidi_math.jl:127-151)
            o = g - 0.5 - np.array(centre)
            u = c / np.linalg.norm(c)
            bb, cc = o @ u, o @ o - radius ** 2
            t = -bb - np.sqrt(bb * bb - cc)
            assert float(qr[k]) == np.float16(t / np.linalg.norm(c))
    # an axis ray 0.5 off the centre line in y and z; a ray that misses; a ray starting inside
    t = ray_sphere_first_hit(np.array([[11.5, 7.5, 7.5], [11.5, 20.0, 7.5], [16.0, 8.0, 8.0]]),
                             np.array([1.0, 0.0, 0.0]), centre, radius)
    assert t[0] == pytest.approx(4.5 - np.sqrt(4.3 ** 2 - 0.5), rel=1e-14)
    assert np.isinf(t[1]) and t[2] == pytest.approx(4.3)


def test_oracle_bouzidi_channel_runs_and_conserves_nothing_spurious():
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    cells, q = sphere_qmap(case.dom, (10.0, 8.0, 8.0), 3.0)
    p = case.params
    p.solid_bc = 3
    p.collect_forces = 0
    d = case.dom
    O = oracle.OracleLevel(d.coords, d.neighbor_table, d.shape, obstacle=d.obstacle)
    O.init_equilibrium(case.rho, case.vel)
    for _ in range(4):
        O.step_bouzidi(p, dict(cells=cells, q=q))
    assert np.isfinite(O.f).all()
    # the sphere sits on the channel axis: the transverse momentum stays at rounding level
    mm = O.mass_momentum()
    assert abs(mm[2]) < 1e-9 * abs(mm[1]) and abs(mm[3]) < 1e-9 * abs(mm[1])


def box_mesh(lo, hi):
    """The 12 triangles of an axis-aligned box."""
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]])
    faces = [(0, 1, 2), (0, 2, 3), (4, 6, 5), (4, 7, 6), (0, 5, 1), (0, 4, 5),
             (3, 2, 6), (3, 6, 7), (0, 3, 7), (0, 7, 4), (1, 5, 6), (1, 6, 2)]
    return np.array([[v[i], v[j], v[k]] for i, j, k in faces])


def test_stl_qmap_of_a_box_matches_the_slab_distances():
    from openaerolab_alpha_01_b200.bouzidi import stl_qmap
    dom = build_box(4, 3, 3)
    lo, hi = np.array([11.3, 9.6, 8.7]), np.array([18.2, 14.45, 15.9])
    gx, gy, gz = dom.cell_positions()
    cen = np.stack([gx - 0.5, gy - 0.5, gz - 0.5], axis=-1)
    dom.obstacle = np.all((cen > lo) & (cen < hi), axis=-1).astype(np.uint8)
    tris = box_mesh(lo - 1.0, hi - 1.0)  # mesh coordinates, shifted back by the offset below
    cells, q, tri = stl_qmap(dom, tris, mesh_offset=(1.0, 1.0, 1.0))
    assert cells.shape[0] > 0
    n_links = 0
    for (b, x, y, z), qr, tr in zip(cells, q, tri):
        o = (dom.coords[b - 1] - 1) * 8 + np.array([x, y, z]) - 0.5
        for k in range(27):
            c = np.array([CX[k], CY[k], CZ[k]], float)
            if qr[k] == 0:
                continue
            n_links += 1
            assert 1 <= tr[k] <= 12
            # entry distance of the ray into the box (slab method), in units of the link
            with np.errstate(divide="ignore", invalid="ignore"):
                t0, t1 = (lo - o) / c, (hi - o) / c
            tn = np.nanmax(np.where(c != 0, np.minimum(t0, t1), -np.inf))
            assert float(qr[k]) == np.float16(tn)
    assert n_links > 100
    # the analytic sphere and a fine triangulation of it give close q values on the same links
    dom2 = build_box(4, 2, 2)
    centre, radius = (16.0, 8.0, 8.0), 4.3
    apply_analytic_sphere_obstacle(dom2, centre, radius)
    th, ph = np.meshgrid(np.linspace(0, np.pi, 61), np.linspace(0, 2 * np.pi, 121), indexing="ij")
    P = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1) * radius + centre
    quads = [(P[i, j], P[i + 1, j], P[i + 1, j + 1], P[i, j + 1]) for i in range(60) for j in range(120)]
    tris = np.array([t for a, b_, c, d in quads for t in ((a, b_, c), (a, c, d))])
    c_s, q_s = sphere_qmap(dom2, centre, radius)
    c_t, q_t, _ = stl_qmap(dom2, tris)
    assert np.array_equal(c_s, c_t)
    both = (q_s > 0) & (q_t > 0)
    assert both.sum() > 0.99 * (q_s > 0).sum()
    assert np.max(np.abs(q_s[both].astype(float) - q_t[both].astype(float))) < 0.02
