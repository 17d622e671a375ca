"""Refined octree meshes on the GPU: the coupled levels against the oracle bit for bit, and the
reference's coupling gates (tools/tests/q19_octree_levels.jl) with its sizes and thresholds:
G2.0 uniform flow through 3 levels, G2.7 interface dissipation of shear waves, G2.3 a vortex
convected across two interfaces, G2.5 mass drift, G2.1 Poiseuille with an interface inside the
channel."""
import math

import numpy as np
import pytest

from .test_gpu_q19 import same_bits
from .test_oracle_q19_levels import (K_FLUID, g25_init, level_fields, oracle_octree, refined_box, refined_slab)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(oal, oracle_lib):
    from openaerolab_alpha_01_b200 import octree
    return oracle_lib, octree


def gpu_state(octree, m, dt, nu, sgs="none", sigma=1.0, body_force=(0.0, 0.0, 0.0)):
    cfg = octree.test_case_config(m.levels[-1], nu_lattice=nu, precision=dt, sgs=sgs, hrr_sigma=sigma,
                                  body_force=body_force)
    return octree.State(m, cfg)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("sgs,sigma,F", [("none", 1.0, (0.0, 0.0, 0.0)), ("wale", 0.98, (0.0, 0.0, 0.0)),
                                         ("vreman", 0.98, (1e-6, 0.0, 2e-6))])
def test_levels_bitwise(env, dt, sgs, sigma, F):
    """Three coupled levels (ghost fills at the half and full time, restrictions, ghost copies) after
    4 coarse steps: every level's state equals the oracle's bit for bit."""
    oracle, octree = env
    m = refined_box(16, 3)
    T, params, _ = oracle_octree(oracle, m, dt, nu=0.004, sgs=sgs, sigma=sigma, body_force=F)
    st = gpu_state(octree, m, dt, 0.004, sgs, sigma, F)
    fields = level_fields(m, g25_init(16), dt)
    T.initialise(params, fields)
    st._upload_levels(fields)
    for l in range(1, 4):
        f, u, rho = st.state(l)
        assert same_bits(f, T.levels[l - 1].f) and same_bits(u, T.levels[l - 1].u)
    for _ in range(2):
        st.advance(2)
        T.advance(params, 2)
        for l in range(1, 4):
            f, u, rho = st.state(l)
            S = T.levels[l - 1]
            assert same_bits(f, S.f), (l, np.abs(f.astype(float) - S.f).max())
            assert same_bits(u, S.u) and same_bits(rho, S.rho)
    assert np.allclose(st.totals(), T.totals(), rtol=1e-12, atol=1e-12)
    st.close()


def test_g20_uniform_flow(env):
    """q19_octree_levels.jl:70-88: a uniform stream through a 3-level refined box, 64 coarse steps."""
    _, octree = env
    m = refined_box(32, 3)
    st = gpu_state(octree, m, np.float64, 0.005)
    U0 = 0.04
    st.initialise(lambda x, y, z: (1.0, U0 + 0 * x, 0 * x, 0 * x))
    st.advance(64)
    worst = worst_rho = 0.0
    for l, lv in enumerate(m.levels, start=1):
        _, u, rho = st.state(l)
        fl = lv.kind == K_FLUID
        uu = u.transpose(0, 2, 1)[fl]
        worst = max(worst, np.abs(uu[:, 0] - U0).max(), np.abs(uu[:, 1:]).max())
        worst_rho = max(worst_rho, np.abs(rho[fl] - 1).max())
    st.close()
    assert worst < 1e-9 and worst_rho < 1e-9, (worst, worst_rho)


def test_g25_mass_drift(env):
    """q19_octree_levels.jl:177-190: 10 n coarse steps of a 3-level refined periodic box, drift < 1e-4."""
    _, octree = env
    n = 32
    m = refined_box(n, 3)
    st = gpu_state(octree, m, np.float64, 0.01)
    st.initialise(g25_init(n))
    m0 = st.mass0
    drift = []
    for s in range(10):
        st.advance(n)
        drift.append((st.total_mass() - m0) / m0)
    assert np.isfinite(st.state(3)[0]).all()
    st.close()
    assert abs(drift[-1]) < 1e-4, drift


def kinetic(st, m):
    """KE over the fluid leaves, each level weighted by its volume in finest cells (no density)."""
    e = 0.0
    L = m.nlevels
    for l, lv in enumerate(m.levels, start=1):
        _, u, _ = st.state(l)
        fl = lv.kind == K_FLUID
        uu = u.transpose(0, 2, 1)[fl].astype(np.float64)
        e += 8.0 ** (L - l) * 0.5 * (uu ** 2).sum()
    return e


def measured_viscosity(st, m, k, steps, levels):
    s1 = steps // 5
    st.advance(s1)
    e1 = kinetic(st, m)
    st.advance(steps - s1)
    e2 = kinetic(st, m)
    return -math.log(e2 / e1) / (2 * k * k * (steps - s1)) / 2 ** (levels - 1)


def test_g27_interface_dissipation(env):
    """q19_octree_levels.jl:90-104: shear waves across and along the interfaces of a refined slab;
    the viscosity of the 2-level run over the mean of the one-level fine and coarse runs, |excess| < 2 %."""
    _, octree = env
    n, nu, A0 = 32, 0.005, 0.01
    k = 2 * math.pi / n
    inits = {"normal": lambda x, y, z: (1.0, A0 * np.sin(k * z), 0 * x, 0 * x),
             "tangential": lambda x, y, z: (1.0, 0 * x, A0 * np.sin(k * x), 0 * x)}
    for name, init in inits.items():
        m = refined_slab(n, 1); s = gpu_state(octree, m, np.float64, nu); s.initialise(init)
        r_f = measured_viscosity(s, m, k, 800, 1); s.close()
        m = refined_slab(n // 2, 1); s = gpu_state(octree, m, np.float64, nu / 2)
        s.initialise(lambda x, y, z: init(2 * x, 2 * y, 2 * z))
        r_c = 2 * measured_viscosity(s, m, 2 * k, 400, 1); s.close()
        m = refined_slab(n, 2); s = gpu_state(octree, m, np.float64, nu); s.initialise(init)
        r_2 = measured_viscosity(s, m, k, 800, 2); s.close()
        excess = (r_2 - 0.5 * (r_f + r_c)) / nu
        assert abs(excess) < 0.02, (name, r_f / nu, r_c / nu, r_2 / nu, excess)


def sampler(st, m):
    states = [st.state(l) for l in range(1, m.nlevels + 1)]

    def at(p):
        l, s = m.locate_leaf(p)
        if l == 0:
            return (np.nan, np.nan, np.nan, np.nan)
        _, u, rho = states[l - 1]
        o, k = s // 8, s % 8
        return float(u[o, 0, k]), float(u[o, 1, k]), float(u[o, 2, k]), float(rho[o, k])
    return at


def test_g23_vortex_across_interfaces(env):
    """q19_octree_levels.jl:106-175: a Taylor vortex convected through the interfaces of a 2-level box
    for one period: swirl peak within 1 % and centroid within 0.01 n of the one-level fine run, far-field
    density noise below 1 % of the core deficit."""
    _, octree = env
    n, U0, umax, rc, nu = 64, 0.04, 0.006, 8.0, 0.005
    res = {}
    for name, nn, levels in (("fine", n, 1), ("coarse", n // 2, 1), ("2-level", n, 2)):
        h = n // nn
        rc_l, nu_l = rc / h, nu / h

        def vortex(x, y, z, c=(nn / 2, nn / 2, nn / 2)):
            dx_ = x - c[0]; dx_ = dx_ - nn * np.round(dx_ / nn)
            dz_ = z - c[2]; dz_ = dz_ - nn * np.round(dz_ / nn)
            r2 = dx_ ** 2 + dz_ ** 2
            e = np.exp(0.5 * (1 - r2 / rc_l ** 2))
            s = umax / rc_l * e
            return 1 - 1.5 * umax ** 2 * e ** 2, U0 - s * dz_, 0 * x, s * dx_

        m = refined_box(nn, levels)
        st = gpu_state(octree, m, np.float64, nu_l)
        st.initialise(vortex)
        steps = round(n / U0 / (h * 2 ** (levels - 1)))
        pts = [(x + 0.5, nn / 2 + 0.5, z + 0.5) for x in range(nn) for z in range(nn)]
        far = []
        for chunk in range(1, 9):
            st.advance(steps // 8)
            xv = (nn / 2 + U0 * (chunk * (steps // 8)) * 2 ** (levels - 1)) % nn
            at = sampler(st, m)
            vals = []
            for p in pts:
                dx_ = p[0] - xv; dx_ -= nn * round(dx_ / nn)
                if math.hypot(dx_, p[2] - nn / 2) > 3 * rc_l:
                    vals.append((at(p)[3] - 1) ** 2)
            far.append(math.sqrt(sum(vals) / len(vals)))
        st.advance(steps - 8 * (steps // 8))
        at = sampler(st, m)
        sw = np.array([math.hypot(at(p)[0] - U0, at(p)[2]) for p in pts])
        P = np.array(pts)
        w = sw ** 2
        res[name] = dict(peak=sw.max(), cx=h * (w * P[:, 0]).sum() / w.sum(), cz=h * (w * P[:, 2]).sum() / w.sum(),
                         far=np.array(far))
        st.close()
    ref, amr = res["fine"], res["2-level"]
    deficit = 1.5 * umax ** 2 * math.e
    noise = (amr["far"] - ref["far"]).max() / deficit
    assert abs(amr["peak"] - ref["peak"]) / ref["peak"] < 0.01, (amr["peak"], ref["peak"])
    assert math.hypot(amr["cx"] - ref["cx"], amr["cz"] - ref["cz"]) < 0.01 * n
    assert noise < 0.01, noise


def test_g21_poiseuille_with_interface(env):
    """q19_octree_levels.jl:194-233: the plates at the finest level, the channel centre one level
    coarser: profile error < 3 %, wall position within 0.1 cells, friction within 2 % (1 and 2 levels)."""
    _, octree = env
    nu, Fx, n, H = 0.1, 1e-5, 48, 16.0
    Lx, Ly, Lz = 24, 2 * n, n
    c = (0.0, Ly / 2 + 0.3, Lz / 2 + 0.2)
    tri = np.concatenate([octree.box_triangles((-Lx, -4 * n, H), (2 * Lx, 4 * n, H + 4 * n)),
                          octree.box_triangles((-Lx, -4 * n, -H - 4 * n), (2 * Lx, 4 * n, -H))])
    tri[..., 1] += c[1]
    tri[..., 2] += c[2]
    for levels in (1, 2):
        spec = octree.MeshSpec(domain=(float(Lx), float(Ly), float(Lz)), periodic=(True, False, False), levels=levels,
                               dx_finest=1.0, band_fine=4, band=3,
                               faces=("periodic", "periodic", "slip", "slip", "slip", "slip"))
        m = octree.generate(tri, spec)
        st = gpu_state(octree, m, np.float64, nu, body_force=(Fx, 0.0, 0.0))
        st.initialise(lambda x, y, z: (1.0, 0 * x, 0 * x, 0 * x))
        steps = round(5 * H ** 2 / nu) // 2 ** (levels - 1)
        st.advance(steps - 1)
        st.advance(1, collect=True)
        at = sampler(st, m)
        d, u, seen = [], [], set()
        for z in range(n):
            p = (Lx / 2 + 0.5, Ly / 2 + 0.5, z + 0.5)
            l, s = m.locate_leaf(p)
            if l == 0 or (l, s) in seen:
                continue
            seen.add((l, s))
            lv = m.levels[l - 1]
            zc = (lv.origin[s // 8, 2] + ((s % 8) >> 2) + 0.5) * lv.dx - c[2]
            if abs(zc) >= H:
                continue
            d.append(zc)
            u.append(at(p)[0])
        d, u = np.array(d), np.array(u)
        A = np.stack([np.ones_like(d), d * d], 1)
        coef = np.linalg.lstsq(A, u, rcond=None)[0]
        H_eff = math.sqrt(-coef[0] / coef[1])
        prof = np.abs(u - Fx / (2 * nu) * (H * H - d * d)).max() / (Fx * H * H / (2 * nu))
        fluid_units = sum(lv.counts["fluid_total"] * 8.0 ** (levels - lv.level) for lv in m.levels)
        fric = abs(abs(st.forces[0]) * 4.0 ** (levels - 1) - Fx * fluid_units) / (Fx * fluid_units)
        st.close()
        assert prof < 0.03 and abs(H_eff - H) < 0.1 and fric < 0.02, (levels, prof, H_eff - H, fric)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_naca_levels_bitwise(env, dt):
    """A small NACA 0012 on 3 levels (cut links and face conditions on the finest level, coupling, WALE
    + HRR): 2 coarse steps equal the oracle bit for bit, per-triangle forces included."""
    oracle, octree = env
    m, cfg = octree.naca_case(chord=32, domain=(256.0, 128.0, 16.0), leading_edge_x=80.0, precision=dt, band_fine=4)
    assert m.counts["leak_cells"] == 0 and m.levels[-1].counts["cut_links"] > 0
    L = m.nlevels
    params = [cfg.params(l, L) for l in range(1, L + 1)]
    descs = [lv.desc() for lv in m.levels]
    T = oracle.OracleQ19Octree(descs, [lv.onbr for lv in m.levels], dt)
    st = octree.State(m, cfg)
    st.initialise_uniform(1.0, cfg.u_lattice, 0.0, 0.0)
    fields = []
    for lv in m.levels:
        u = np.zeros((lv.nocts, 3, 8), dt)
        u[:, 0] = dt(cfg.u_lattice)
        fields.append((np.ones((lv.nocts, 8), dt), u, None))
    T.initialise(params, fields)
    st.advance(1)
    T.advance(params, 1)
    st.advance(1, collect=True)
    T.advance(params, 1, collect=True)
    for l in range(1, L + 1):
        f, u, rho = st.state(l)
        S = T.levels[l - 1]
        assert same_bits(f, S.f) and same_bits(u, S.u) and same_bits(rho, S.rho), l
    assert same_bits(st.forces_per_triangle(), T.per_tri)
    assert np.allclose(st.forces, T.forces, rtol=1e-12, atol=1e-15)
    st.close()
