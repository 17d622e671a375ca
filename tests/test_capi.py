"""The C-ABI library loads, exports every symbol include/oal.h declares, and its host-side
logic (operator registry, defaults, domain builders) matches the reference semantics and the
oracle bit for bit. No compute call here needs a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200 import solver

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "oal.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(oal_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(oal):
    L = C.CDLL(str(capi.LIB_PATH))
    syms = header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(capi.exported_symbols()) == syms


def test_abi_and_status_strings(oal):
    L = capi.lib()
    assert L.oal_abi_version() == capi.OAL_ABI_VERSION
    assert L.oal_status_string(capi.OAL_E_UNKNOWN_OPERATOR) == b"unknown collision operator"


def test_operator_registry(oal):
    # physics_kernels.jl:50-75: :cumulant (D3Q27), :entropic (D3Q39); anything else errors
    assert solver.get_collision_kernel("cumulant") == capi.OAL_OP_CUMULANT_D3Q27
    assert solver.get_collision_kernel(":cumulant") == capi.OAL_OP_CUMULANT_D3Q27
    assert solver.get_collision_kernel("entropic") == capi.OAL_OP_ENTROPIC_D3Q39
    assert solver.get_collision_kernel("hrr") == capi.OAL_OP_HRR_D3Q19
    with pytest.raises(capi.OALError) as e:
        solver.get_collision_kernel("regularized_bgk")
    assert e.value.status == capi.OAL_E_UNKNOWN_OPERATOR
    assert "Valid options" in str(e.value)


def test_default_params_follow_config_loader(oal):
    p = capi.default_params()
    assert p.abi_version == 1 and p.operator_id == capi.OAL_OP_CUMULANT_D3Q27
    assert abs(p.c_wale - 0.20) < 1e-7 and p.nu_sgs_background == 0.0
    assert p.omega_bulk == 1 and p.omega3 == 1 and p.omega4 == 1
    assert p.adaptive_omega4 == 1 and abs(p.lambda_param - 1 / 6) < 1e-7
    assert p.limiter_type == capi.OAL_LIMITER_FACTORED and p.compressible_corr == 0
    assert p.wall_model_active == 0 and p.wall_model_max_distance == 10.0
    assert C.sizeof(capi.StepParams) == 4 * len(capi.StepParams._fields_) == 160  # 40 four-byte scalars
    assert p.svv_x_epsilon == 0.0 and p.svv_yz_epsilon == 0.0  # SVV off (config_loader.jl:660-669)


@pytest.mark.parametrize("dims,mask", [((2, 2, 2), 7), ((4, 2, 3), 0), ((3, 1, 2), 2), ((1, 1, 1), 7), ((5, 3, 2), 5)])
def test_box_blocks_match_oracle(oal, oracle_lib, dims, mask):
    dom = solver.build_box(*dims, periodic=(bool(mask & 1), bool(mask & 2), bool(mask & 4)))
    coords, nbr = oracle_lib.build_box(*dims, mask)
    assert np.array_equal(dom.coords, coords)
    assert np.array_equal(dom.neighbor_table, nbr)
    n = coords.shape[0]
    # self entry and symmetry: b -> a in direction d  <=>  a -> b in direction 26 - d
    assert np.array_equal(nbr[13], np.arange(1, n + 1))
    for d in range(27):
        for b in range(n):
            a = nbr[d, b]
            if a > 0 and not (dims[0] == 1 or dims[1] == 1 or dims[2] == 1):
                assert nbr[26 - d, a - 1] == b + 1


def test_sphere_matches_oracle(oal, oracle_lib):
    dom = solver.build_box(8, 4, 4)
    n = solver.apply_analytic_sphere_obstacle(dom, (32.0, 16.0, 16.0), 12.0)
    obst, n2 = oracle_lib.sphere(dom.coords, (32.0, 16.0, 16.0), 12.0)
    assert n == n2 and np.array_equal(dom.obstacle, obst)
    assert abs(n - 4 / 3 * np.pi * 12 ** 3) / n < 0.02


def test_geometry_without_device_reports_no_device(oal):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    dom = solver.build_box(2, 2, 2, periodic=(True, True, True))
    with pytest.raises(capi.OALError) as e:
        solver.Geometry(dom)
    assert e.value.status == capi.OAL_E_NO_DEVICE
