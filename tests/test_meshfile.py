"""The reference's octree mesh file (octree.jl:158-233): a generated mesh written and read back
field by field, the SHA-256 trailer and header checks, and on the GPU the same steps from the
generated and from the read mesh."""
import numpy as np
import pytest

FIELDS = ("origin", "real", "kind", "face", "onbr", "cutidx", "special", "cut_slot", "cut_off", "cut_dir", "cut_q",
          "cut_tri", "cut_partner", "ghost_slot", "ghost_donor", "ghost_w", "restrict_slot", "restrict_src",
          "restrict_cubic")


def refined_mesh_with_body():
    from openaerolab_alpha_01_b200 import octree
    L = 32.0
    tri = octree.box_triangles((12.0, 12.0, 12.0), (20.0, 20.0, 20.0))
    spec = octree.MeshSpec(domain=(L, L, L), periodic=(False, False, False), levels=2, dx_finest=1.0,
                           surface_level=2, band_fine=3, band=2,
                           faces=("inlet", "outlet", "slip", "slip", "slip", "slip"))
    return octree.generate(tri, spec), tri


def test_round_trip_and_checks(oal, tmp_path):
    from openaerolab_alpha_01_b200 import octree
    m, tri = refined_mesh_with_body()
    p = tmp_path / "mesh.oct"
    digest = octree.write_mesh(p, m, tri, offset=(0.5, 0.0, -1.0), config_sha="cfg", stl_sha="stl")
    raw = p.read_bytes()
    import hashlib
    assert hashlib.sha256(raw[:-32]).hexdigest() == digest and raw[:8] == b"OCTQ19M\0"
    assert np.frombuffer(raw[8:16], "<i8")[0] == 5
    r = octree.read_mesh(p, faces=("inlet", "outlet", "slip", "slip", "slip", "slip"))
    assert r.nlevels == m.nlevels and r.spec.domain == m.spec.domain and r.offset == (0.5, 0.0, -1.0)
    assert r.config_sha == "cfg" and r.stl_sha == "stl" and np.array_equal(r.triangles, np.asarray(tri).reshape(-1, 3, 3))
    assert r.counts["per_level"] == m.counts["per_level"]
    for a, b in zip(m.levels, r.levels):
        assert (a.level, a.dx, a.n, a.nocts, a.faces, a.ntri) == (b.level, b.dx, b.n, b.nocts, b.faces, b.ntri)
        for f in FIELDS:
            x, y = getattr(a, f), getattr(b, f)
            assert x.shape == y.shape and np.array_equal(x, y), f
    # a changed byte fails the trailer; another magic or format is refused
    bad = bytearray(raw)
    bad[100] ^= 1
    (tmp_path / "bad.oct").write_bytes(bytes(bad))
    with pytest.raises(ValueError):
        octree.read_mesh(tmp_path / "bad.oct")
    body = bytearray(raw[:-32])
    body[8:16] = np.array([4], "<i8").tobytes()
    (tmp_path / "old.oct").write_bytes(bytes(body) + hashlib.sha256(bytes(body)).digest())
    with pytest.raises(ValueError):
        octree.read_mesh(tmp_path / "old.oct")


@pytest.mark.gpu
def test_read_mesh_steps_like_the_generated_one(oal, tmp_path):
    """A mesh read from the file steps bit for bit like the mesh it was written from."""
    from openaerolab_alpha_01_b200 import octree
    m, tri = refined_mesh_with_body()
    octree.write_mesh(tmp_path / "m.oct", m, tri)
    r = octree.read_mesh(tmp_path / "m.oct", faces=("inlet", "outlet", "slip", "slip", "slip", "slip"))
    out = []
    for mesh in (m, r):
        cfg = octree.CaseConfig(nu_lattice=0.01, u_lattice=0.05, dx=1.0)
        st = octree.State(mesh, cfg, precision=np.float32)
        st.initialise_uniform(1.0, 0.05, 0.0, 0.0)
        st.advance(6)
        out.append([st.state(l) for l in range(1, mesh.nlevels + 1)])
        st.close()
    for la, lb in zip(out[0], out[1]):
        for x, y in zip(la, lb):
            assert np.array_equal(x, y)
