"""The reference's raw state dump, written and read (src/io/raw_state_dump.jl:1-48).

The reference writes the macroscopic state of every level as little-endian binaries,
``<output_dir>/raw_state/step_<NNNNNN>/level_<L>.bin``, laid out as

    Int32   magic 0x4C424D31 ("LBM1")
    Int32   level_id, n_blocks, block_size, grid_dim_x, grid_dim_y, grid_dim_z
    Float64 dx
    Int32   coords[3, n_blocks]          (bx, by, bz) of each block, 1-based
    Float32 rho[bs, bs, bs, n_blocks]
    Float32 vel[bs, bs, bs, n_blocks, 3]
    UInt8   obstacle[bs, bs, bs, n_blocks]  (1 = solid)

with Julia's column-major order (x fastest). This library's host arrays are in the same element
order: coords (n_blocks, 3), rho (n_blocks, 512), vel (3, n_blocks, 512), obstacle (n_blocks, 512)
in C order, cell = x + 8 y + 64 z. So a level of this library can be dumped for the reference's
readers, and a reference dump read back as this library's arrays.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

MAGIC = 0x4C424D31
BLOCK_SIZE = 8


def write_level(path, level_id: int, coords, grid_dim, dx: float, rho, vel, obstacle=None) -> None:
    """Write one level file. coords (n_blocks, 3) 1-based block coordinates; grid_dim the blocks
    along x, y, z; rho (n_blocks, 512); vel (3, n_blocks, 512); obstacle (n_blocks, 512) or None
    (no solid cell)."""
    coords = np.asarray(coords)
    nb = coords.shape[0]
    if coords.shape != (nb, 3):
        raise ValueError("coords must be (n_blocks, 3)")
    rho = np.asarray(rho).reshape(nb, 512)
    vel = np.asarray(vel).reshape(3, nb, 512)
    obst = np.zeros((nb, 512), np.uint8) if obstacle is None else (np.asarray(obstacle).reshape(nb, 512) != 0)
    header = np.array([MAGIC, level_id, nb, BLOCK_SIZE, *grid_dim], dtype="<i4")
    with open(path, "wb") as io:
        io.write(header.tobytes())
        io.write(np.array([dx], dtype="<f8").tobytes())
        io.write(np.ascontiguousarray(coords, dtype="<i4").tobytes())
        io.write(np.ascontiguousarray(rho, dtype="<f4").tobytes())
        io.write(np.ascontiguousarray(vel, dtype="<f4").tobytes())
        io.write(np.ascontiguousarray(obst, dtype=np.uint8).tobytes())


def read_level(path) -> dict:
    """Read one level file (this library's writer or the reference's) into this library's arrays."""
    data = Path(path).read_bytes()
    head = np.frombuffer(data, dtype="<i4", count=7)
    if int(head[0]) != MAGIC:
        raise ValueError(f"{path}: not a raw state file (magic {int(head[0]):#x})")
    level_id, nb, bs = int(head[1]), int(head[2]), int(head[3])
    if bs != BLOCK_SIZE:
        raise ValueError(f"{path}: block size {bs}, this library uses {BLOCK_SIZE}")
    off = 28
    dx = float(np.frombuffer(data, dtype="<f8", count=1, offset=off)[0]); off += 8
    ncell = nb * bs ** 3
    need = off + 12 * nb + 4 * ncell + 12 * ncell + ncell
    if len(data) != need:
        raise ValueError(f"{path}: {len(data)} bytes, {need} expected for {nb} blocks")
    coords = np.frombuffer(data, dtype="<i4", count=3 * nb, offset=off).reshape(nb, 3).copy(); off += 12 * nb
    rho = np.frombuffer(data, dtype="<f4", count=ncell, offset=off).reshape(nb, 512).copy(); off += 4 * ncell
    vel = np.frombuffer(data, dtype="<f4", count=3 * ncell, offset=off).reshape(3, nb, 512).copy(); off += 12 * ncell
    obstacle = np.frombuffer(data, dtype=np.uint8, count=ncell, offset=off).reshape(nb, 512).copy()
    return {"level_id": level_id, "n_blocks": nb, "block_size": bs, "grid_dim": tuple(int(v) for v in head[4:7]),
            "dx": dx, "coords": coords, "rho": rho, "vel": vel, "obstacle": obstacle}


def step_dir(output_dir, step: int) -> Path:
    return Path(output_dir) / "raw_state" / f"step_{step:06d}"


def dump_raw_state(levels, output_dir, step: int) -> Path:
    """Dump levels the way the reference's dump_raw_state does for one step. `levels` holds
    (level_id, domain, rho, vel, dx) tuples, domain a solver.BlockDomain (its coords, block grid and
    obstacle). Returns the step directory."""
    d = step_dir(output_dir, step)
    os.makedirs(d, exist_ok=True)
    for level_id, dom, rho, vel, dx in levels:
        write_level(d / f"level_{level_id}.bin", level_id, dom.coords, (dom.bx_max, dom.by_max, dom.bz_max), dx,
                    rho, vel, dom.obstacle)
    return d


def dump_level(level, dom, output_dir, step: int, level_id: int = 1, dx: float = 1.0) -> Path:
    """Dump the macroscopic state of one solver.Level (its density and velocity outputs)."""
    _, rho, vel = level.state()
    return dump_raw_state([(level_id, dom, rho, vel, dx)], output_dir, step)


def dump_hierarchy(hierarchy, domains, output_dir, step: int) -> Path:
    """Dump every level of an amr.Hierarchy; level l (0 = coarsest) is the reference's level_id l + 1
    with dx = 2^-l of the coarse cell."""
    rows = []
    for l, dom in enumerate(domains):
        _, rho, vel = hierarchy.level(l).state()
        rows.append((l + 1, dom, rho, vel, 0.5 ** l))
    return dump_raw_state(rows, output_dir, step)
