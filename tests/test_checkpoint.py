"""Octree checkpoints (write_checkpoint! / read_checkpoint! / resume_checkpoint!,
src/octree_q19/src/io_run.jl:274-323).

CPU: the byte layout (header offsets, both buffers per level, tau_w, no trailer), the round trip,
and each of the reader's refusals. GPU: a run checkpointed after n steps and resumed into a fresh
state continues bit for bit like the uninterrupted run (one level and a refined three-level mesh),
and the writer keeps the newest `keep` files.
"""
import numpy as np
import pytest

from openaerolab_alpha_01_b200 import octree

HEADER = 8 + 8 + 8 + 64 + 64 + 8 + 8 + 8 + 8 + 9 * 8 + 8  # magic .. level count


def levels(rng, sizes, dt, ncut=(0, 0)):
    out = []
    for no, nc in zip(sizes, ncut):
        out.append({"f": rng.random((no, 19, 8)).astype(dt), "g": rng.random((no, 19, 8)).astype(dt),
                    "u": rng.random((no, 3, 8)).astype(dt), "v": rng.random((no, 3, 8)).astype(dt),
                    "rho": rng.random((no, 8)).astype(dt), "rhob": rng.random((no, 8)).astype(dt),
                    "tau_w": rng.random(nc).astype(dt)})
    return out


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_layout_and_round_trip(dt):
    rng = np.random.default_rng(3)
    lv = levels(rng, (5, 3), dt, (4, 0))
    sums = np.arange(9, dtype=np.float64)
    data = octree.pack_checkpoint(lv, dt, 1234, 0.04, 512.5, 7, sums, "abc", "d" * 70)
    s = np.dtype(dt).itemsize
    per = [8 + no * (2 * 19 * 8 + 2 * 3 * 8 + 2 * 8) * s + 8 + nc * s for no, nc in ((5, 4), (3, 0))]
    assert len(data) == HEADER + sum(per)
    assert data[:8] == b"OCTQ19C\0"
    assert np.frombuffer(data[8:24], "<i8").tolist() == [1, s]
    assert data[24:88] == b"abc" + b" " * 61 and data[88:152] == b"d" * 64
    assert np.frombuffer(data[152:160], "<i8")[0] == 1234
    assert np.frombuffer(data[160:176], "<f8").tolist() == [0.04, 512.5]
    assert np.frombuffer(data[176:184], "<i8")[0] == 7
    assert np.array_equal(np.frombuffer(data[184:256], "<f8"), sums)
    assert np.frombuffer(data[256:264], "<i8")[0] == 2
    assert np.frombuffer(data[264:272], "<i8")[0] == 5
    # the first array is level 1's f, in the reference's column-major (8, 19, nocts) order
    f1 = np.frombuffer(data[272:272 + 5 * 19 * 8 * s], np.dtype(dt).newbyteorder("<"))
    assert np.array_equal(f1.reshape(5, 19, 8), lv[0]["f"])
    ck = octree.unpack_checkpoint(data, dt, "abc", "d" * 64, [5, 3], [4, 0])
    assert ck["step"] == 1234 and ck["n_avg"] == 7 and ck["mass0"] == 512.5
    assert np.array_equal(ck["sums"], sums)
    for a, b in zip(ck["levels"], lv):
        for k in b:
            assert np.array_equal(a[k], b[k]), k


def test_reader_refusals():
    rng = np.random.default_rng(4)
    lv = levels(rng, (2,), np.float32, (1,))
    data = octree.pack_checkpoint(lv, np.float32, 10, 0.05, 1.0, config_sha="cfg", stl_sha="stl")
    cases = [
        (b"X" + data[1:], {}, "not a checkpoint"),
        (data[:8] + np.array([2], "<i8").tobytes() + data[16:], {}, "checkpoint format"),
        (data, dict(precision=np.float64), "precision"),
        (data, dict(config_sha="other"), "another case"),
        (data, dict(stl_sha="other"), "another case"),
        (data, dict(octs=[2, 1]), "level count"),
        (data, dict(octs=[3]), "oct count"),
        (data, dict(ncut=[0]), "wall-model size"),
        (data + b"\0", {}, "trailing data"),
        (data[:-3], {}, "ends early"),
    ]
    for blob, kw, msg in cases:
        with pytest.raises(ValueError, match=msg):
            octree.unpack_checkpoint(blob, **kw)
    assert octree.unpack_checkpoint(data, np.float32, "cfg", "stl", [2], [1])["step"] == 10


def _tgv(dx_box=16):
    return lambda x, y, z: (1.0 + 0 * x, 0.04 * np.sin(2 * np.pi * x / dx_box) * np.cos(2 * np.pi * y / dx_box),
                            -0.04 * np.cos(2 * np.pi * x / dx_box) * np.sin(2 * np.pi * y / dx_box), 0 * x)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [np.float32, np.float64])
def test_resume_continues_bit_for_bit(oal, tmp_path, precision):
    box = octree.PeriodicBox(16, 16, 8)
    cfg = octree.test_case_config(box, nu_lattice=0.02, u_lattice=0.04)
    cfg.sgs, cfg.hrr_sigma, cfg.precision = "wale", 0.98, precision
    A = octree.State(box, cfg).initialise(_tgv())
    A.advance(7)
    path = octree.write_checkpoint(A, tmp_path, n_avg=3, sums=np.ones(9))
    A.advance(9)
    B = octree.State(box, cfg).initialise_uniform(1.0, 0.0, 0.0, 0.0)
    assert octree.resume_checkpoint(B, tmp_path) == 7
    assert B.mass0 == A.mass0
    B.advance(9)
    for a, b in zip(A.state(), B.state()):
        assert np.array_equal(a, b)
    assert path.endswith("checkpoint_000000007.bin")
    A.close(); B.close()


@pytest.mark.gpu
def test_refined_mesh_resume_and_keep(oal, tmp_path):
    L = 32.0
    tri = octree.box_triangles((12.0, 12.0, 12.0), (20.0, 20.0, 20.0))
    spec = octree.MeshSpec(domain=(L, L, L), periodic=(False, False, False), levels=2, dx_finest=1.0,
                           surface_level=2, band_fine=3, band=2,
                           faces=("inlet", "outlet", "slip", "slip", "slip", "slip"))
    mesh = octree.generate(tri, spec)
    cfg = octree.CaseConfig(nu_lattice=0.01, u_lattice=0.05, dx=1.0)
    A = octree.State(mesh, cfg, precision=np.float32).initialise_uniform(1.0, 0.05, 0.0, 0.0)
    for n in (2, 2, 2):
        A.advance(n)
        octree.write_checkpoint(A, tmp_path, keep=2)
    files = sorted(p.name for p in (tmp_path / "checkpoints").iterdir())
    assert files == ["checkpoint_000000004.bin", "checkpoint_000000006.bin"]
    A.advance(3)
    B = octree.State(mesh, cfg, precision=np.float32).initialise_uniform(1.0, 0.0, 0.0, 0.0)
    assert octree.resume_checkpoint(B, tmp_path) == 6
    B.advance(3)
    for l in range(1, mesh.nlevels + 1):
        for a, b in zip(A.state(l), B.state(l)):
            assert np.array_equal(a, b)
    box = octree.PeriodicBox(8, 8, 8)
    other = octree.State(box, octree.test_case_config(box))
    with pytest.raises(ValueError):
        octree.resume_checkpoint(other, tmp_path)
    A.close(); B.close(); other.close()
