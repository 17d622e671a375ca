"""Generates tests/golden/oracle_channel_fp64.json: the CPU oracle on a small sphere channel
(inlet / zero-gradient outlet / lateral mirrors, half-way walls with momentum exchange, FP64).

The reference (Julia) cannot run here, so this fixture pins the oracle restatement against its
own later changes; it is not a reference-produced vector.

    python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def channel_case(oracle, steps=30):
    from openaerolab_alpha_01_b200 import _capi as capi
    bx, by, bz = 4, 2, 2
    coords, nbr = oracle.build_box(bx, by, bz, 0)
    obst, n_solid = oracle.sphere(coords, (10.0, 8.0, 8.0), 3.0)
    nb = coords.shape[0]
    L = oracle.OracleLevel(coords, nbr, (8 * bx, 8 * by, 8 * bz), obstacle=obst)
    vel = np.zeros((3, nb, 512))
    vel[0] = np.where(obst != 0, 0.0, 0.05)
    L.init_equilibrium(np.ones((nb, 512)), vel)
    p = capi.default_params(tau=0.53, c_wale=0.2, u_inlet=0.05, solid_bc=capi.OAL_SOLID_HALFWAY, collect_forces=1)
    for _ in range(steps):
        L.step(p)
    probe = L.f[:, 5, ::37].ravel()
    return dict(n_solid=n_solid, force=L.force.tolist(), mass_momentum=L.mass_momentum().tolist(),
                probe_f=probe.tolist())


if __name__ == "__main__":
    import oracle
    oracle.build()
    out = channel_case(oracle)
    (Path(__file__).parent / "oracle_channel_fp64.json").write_text(json.dumps(out, indent=1))
    print("force", out["force"], "solid", out["n_solid"])
