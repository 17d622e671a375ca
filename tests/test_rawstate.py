"""The reference's raw state dump format (src/io/raw_state_dump.jl:1-48): header fields at their
byte offsets, element order of each array, round trip; on the GPU, a level's state dumped and read
back."""
import numpy as np
import pytest

from openaerolab_alpha_01_b200 import rawstate
from openaerolab_alpha_01_b200.solver import apply_analytic_sphere_obstacle, build_box


def _arrays(dom, seed=0):
    rng = np.random.default_rng(seed)
    nb = dom.n_blocks
    return rng.random((nb, 512)).astype(np.float32), rng.standard_normal((3, nb, 512)).astype(np.float32)


def test_layout_and_round_trip(tmp_path):
    dom = build_box(2, 1, 3)
    apply_analytic_sphere_obstacle(dom, (8.0, 4.0, 12.0), 3.0)
    rho, vel = _arrays(dom)
    d = rawstate.dump_raw_state([(2, dom, rho, vel, 0.25)], tmp_path, 17)
    path = d / "level_2.bin"
    assert d == tmp_path / "raw_state" / "step_000017"
    raw = path.read_bytes()
    nb = dom.n_blocks
    # header: magic, level_id, n_blocks, block_size, grid dims, then dx
    assert np.frombuffer(raw[:28], "<i4").tolist() == [0x4C424D31, 2, nb, 8, 2, 1, 3]
    assert np.frombuffer(raw[28:36], "<f8")[0] == 0.25
    # coords[3, n] column-major: (bx, by, bz) of block 1, then block 2, ...
    c = np.frombuffer(raw[36:36 + 12 * nb], "<i4")
    assert c[:3].tolist() == dom.coords[0].tolist() and c[3:6].tolist() == dom.coords[1].tolist()
    # rho[x, y, z, b]: x fastest, then y, z, block
    r0 = 36 + 12 * nb
    r = np.frombuffer(raw[r0:r0 + 4 * 512 * nb], "<f4")
    assert r[1] == rho[0, 1] and r[8] == rho[0, 8] and r[512] == rho[1, 0]
    # vel[x, y, z, b, c]: the component slowest
    v0 = r0 + 4 * 512 * nb
    v = np.frombuffer(raw[v0:v0 + 12 * 512 * nb], "<f4")
    assert v[512 * nb] == vel[1, 0, 0] and v[2 * 512 * nb + 3] == vel[2, 0, 3]
    assert len(raw) == v0 + 12 * 512 * nb + 512 * nb
    back = rawstate.read_level(path)
    assert back["level_id"] == 2 and back["grid_dim"] == (2, 1, 3) and back["dx"] == 0.25
    assert np.array_equal(back["coords"], dom.coords)
    assert np.array_equal(back["rho"], rho) and np.array_equal(back["vel"], vel)
    assert np.array_equal(back["obstacle"], (dom.obstacle != 0).astype(np.uint8))


def test_rejects_other_files(tmp_path):
    p = tmp_path / "x.bin"
    p.write_bytes(np.array([1, 2, 3, 8, 1, 1, 1], "<i4").tobytes() + b"\0" * 8)
    with pytest.raises(ValueError):
        rawstate.read_level(p)
    dom = build_box(1, 1, 1)
    rho, vel = _arrays(dom)
    rawstate.write_level(p, 1, dom.coords, (1, 1, 1), 1.0, rho, vel)
    p.write_bytes(p.read_bytes()[:-5])
    with pytest.raises(ValueError):
        rawstate.read_level(p)


@pytest.mark.gpu
def test_level_dump_matches_state(oal, tmp_path):
    from openaerolab_alpha_01_b200.cases import sphere_channel_case
    from openaerolab_alpha_01_b200.solver import Geometry, Level
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    g = Geometry(case.dom)
    L = Level(g, storage="f16")
    L.init_equilibrium(case.rho, case.vel)
    L.execute_timestep_batch(case.params, 5)
    d = rawstate.dump_level(L, case.dom, tmp_path, 5)
    back = rawstate.read_level(d / "level_1.bin")
    _, rho, vel = L.state()
    assert np.array_equal(back["rho"], rho.astype(np.float32)) and np.array_equal(back["vel"], vel.astype(np.float32))
    assert back["obstacle"].sum() == int((case.dom.obstacle != 0).sum())
    L.close()
    g.close()
