"""Sealed cavities in the octree generator (MeshSpec seal_cavities, generator.jl:383-414,
geometry.jl:275-295), the reference's test "sealed cavities: a sphere with its top cap missing"
(tools/tests/q19_octree_generator.jl:137-160) with its case and thresholds: a sphere of diameter 1
m in a 6 x 4 x 4 m domain on 3 levels (finest 0.025 m) with the triangles above z = c + 0.42
removed. Without sealing the fill floods the interior through the hole and the leak check reports
it; with sealing the interior stays solid and the exterior is unchanged. Host code only."""
import math

import numpy as np
import pytest

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200 import octree


def sphere_tris(n_lat, n_lon, r=0.5, c=(0.0, 0.0, 0.0)):
    """The latitude-longitude tessellation of the reference's geometry helpers."""
    P = lambda t, f: (c[0] + r * math.sin(t) * math.cos(f), c[1] + r * math.sin(t) * math.sin(f), c[2] + r * math.cos(t))
    out = []
    for i in range(n_lat):
        for j in range(n_lon):
            t0, t1 = math.pi * i / n_lat, math.pi * (i + 1) / n_lat
            f0, f1 = 2 * math.pi * j / n_lon, 2 * math.pi * (j + 1) / n_lon
            a, b, cc, d = P(t0, f0), P(t1, f0), P(t1, f1), P(t0, f1)
            if i < n_lat - 1:
                out.append((a, b, cc))
            if i > 0:
                out.append((a, cc, d))
    return np.array(out)


def kind_at(m, p):
    l, s = m.locate_leaf(p)
    assert l > 0
    return int(m.levels[l - 1].kind[s // 8, s % 8])


def volumes(m, key):
    return sum(lv.counts[key] * lv.dx ** 3 for lv in m.levels)


@pytest.fixture(scope="module")
def meshes(oal):
    tri = sphere_tris(24, 48, c=(2.0, 2.0, 2.0))
    tri_h = np.array([t for t in tri if not all(v[2] > 2.42 for v in t)])
    assert len(tri_h) < len(tri)
    spec = dict(domain=(6.0, 4.0, 4.0), levels=3, dx_finest=0.025, band_fine=4, band=3)
    closed = octree.generate(tri, octree.MeshSpec(**spec))
    open_ = octree.generate(tri_h, octree.MeshSpec(**spec))
    sealed = octree.generate(tri_h, octree.MeshSpec(seal_cavities=True, **spec))
    return closed, open_, sealed


def test_open_sphere_floods(meshes):
    _, m, _ = meshes
    assert kind_at(m, (2.0, 2.0, 2.0)) == capi.OAL_Q19_K_FLUID
    assert m.counts["leak_cells"] > 0
    assert m.counts["sealed_cells"] == 0


def test_sealed_interior_stays_solid(meshes):
    closed, _, m = meshes
    assert m.counts["sealed_cells"] > 0 and m.counts["leak_cells"] == 0
    assert kind_at(m, (2.0, 2.0, 2.0)) == capi.OAL_Q19_K_SOLID
    assert kind_at(m, (2.0, 2.0, 2.9)) == capi.OAL_Q19_K_FLUID
    assert kind_at(m, (1.3, 2.0, 2.0)) == capi.OAL_Q19_K_FLUID
    assert volumes(m, "solid") == pytest.approx(math.pi / 6, rel=0.03)
    assert volumes(m, "fluid_total") == pytest.approx(6 * 4 * 4 - math.pi / 6, rel=0.01)
    f_closed = sum(lv.counts["fluid_total"] for lv in closed.levels)
    f_sealed = sum(lv.counts["fluid_total"] for lv in m.levels)
    assert abs(f_sealed - f_closed) < 0.02 * f_closed


def test_sealing_leaves_a_closed_body_alone(meshes, oal):
    closed, _, _ = meshes
    tri = sphere_tris(24, 48, c=(2.0, 2.0, 2.0))
    m = octree.generate(tri, octree.MeshSpec(domain=(6.0, 4.0, 4.0), levels=3, dx_finest=0.025, band_fine=4, band=3,
                                             seal_cavities=True))
    # the sealed slots of a closed body are the ones the fill would not reach anyway
    for a, b in zip(closed.levels, m.levels):
        assert np.array_equal(a.kind, b.kind)
    assert m.counts["leak_cells"] == 0


def test_per_box_surface_levels(oal):
    """SurfaceLevel boxes (generator.jl:18-21, 185): the surface band reaches the box's level only
    for cells whose centre lies in the box; elsewhere the global surface level holds."""
    tri = sphere_tris(24, 48, c=(2.0, 2.0, 2.0))
    base = dict(domain=(6.0, 4.0, 4.0), levels=3, dx_finest=0.025, band_fine=4, band=3, surface_level=2)
    coarse = octree.generate(tri, octree.MeshSpec(**base))
    assert coarse.levels[2].counts["fluid_total"] == 0
    box = octree.SurfaceLevel(3, (1.0, 1.0, 2.0), (3.0, 3.0, 3.0))   # the upper half of the sphere
    m = octree.generate(tri, octree.MeshSpec(surface_levels=(box,), **base))
    fine = m.levels[2]
    assert fine.counts["fluid_total"] > 0
    # the finest level's cells hug the upper half: their centres lie above the box's floor, less a
    # band and the 2:1 buffers of the coarser levels
    cells = fine.slot_centres().transpose(0, 2, 1).reshape(-1, 3)[fine.kind.reshape(-1) == capi.OAL_Q19_K_FLUID]
    assert cells[:, 2].min() > 2.0 - 0.5 and cells[:, 2].max() < 3.0
    # a box of the global level changes nothing
    same = octree.generate(tri, octree.MeshSpec(surface_levels=(octree.SurfaceLevel(2, (0, 0, 0), (6, 4, 4)),), **base))
    for a, b in zip(coarse.levels, same.levels):
        assert np.array_equal(a.kind, b.kind)
    with pytest.raises(capi.OALError):
        octree.generate(tri, octree.MeshSpec(surface_levels=(octree.SurfaceLevel(4, (0, 0, 0), (1, 1, 1)),), **base))
