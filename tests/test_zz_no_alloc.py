"""The no-allocation entry point (oal_mass_momentum_noalloc) against the level's own FP64
mass/momentum reduction (oal_level_mass_momentum) on the same device state.

The entry point is for callers that cannot call cudaMalloc when they need conservation totals
(a stream-ordered pool that forbids stray allocations, a host runtime that must not grow device
memory between steps); its scratch is a fixed device array inside the library. This file is collected last so that a failure here stops a `-x` run only after
every other test ran; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from openaerolab_alpha_01_b200 import _capi as capi
from openaerolab_alpha_01_b200.cases import sphere_channel_case, taylor_green_case
from openaerolab_alpha_01_b200.solver import Geometry, Level

RTOL = 1e-12  # both are FP64 sums of the same values in the same order


def _noalloc(L, obstacle_dev, out_dev, n_blocks):
    """The caller's own copy of the level's populations, in the reference layout (8,8,8,nb,27),
    FP32 (exactly the decoded values the level sums), reduced without allocation."""
    import torch
    f, _, _ = L.state()
    fd = torch.tensor(f, dtype=torch.float32, device="cuda").contiguous()
    capi.check(capi.lib().oal_mass_momentum_noalloc(fd.data_ptr(), capi.OAL_STORE_F32, 512, 512 * n_blocks,
                                                    None if obstacle_dev is None else obstacle_dev.data_ptr(),
                                                    n_blocks, out_dev.data_ptr(), None))
    torch.cuda.synchronize()
    del fd


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_noalloc_matches_level_reduction_twice(oal, storage):
    import torch
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    g = Geometry(case.dom)
    L = Level(g, storage=storage)
    L.init_equilibrium(case.rho, case.vel)
    obst = torch.tensor(case.dom.obstacle, dtype=torch.uint8, device="cuda").contiguous()
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row; the second reuses the shared scratch
        for _ in range(3):
            L.perform_timestep(case.params)
        expect = L.mass_momentum()
        out.fill_(np.nan)
        _noalloc(L, obst, out, case.dom.n_blocks)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, expect, rtol=RTOL, atol=1e-12 * abs(expect[0]))
    L.close()
    g.close()


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64"])
def test_noalloc_on_the_level_buffer_in_its_stored_type(oal, storage):
    """The level's own population buffer (block-major, stored type, the level's strides) handed
    to the entry point: every storage branch of the reduction runs on the GPU."""
    import torch
    case = sphere_channel_case(32, 16, 16, diameter=6.0, centre_x=10.0, u_inlet=0.05, re=100.0)
    g = Geometry(case.dom)
    L = Level(g, storage=storage, layout="block")
    L.init_equilibrium(case.rho, case.vel)
    for _ in range(4):
        L.perform_timestep(case.params)
    lay = L.layout()
    f_dev = C.c_void_p()
    capi.check(capi.lib().oal_level_device_state(L.handle, C.byref(f_dev), None, None))
    obst = torch.tensor(case.dom.obstacle, dtype=torch.uint8, device="cuda").contiguous()
    out = torch.full((4,), np.nan, dtype=torch.float64, device="cuda")
    capi.check(capi.lib().oal_mass_momentum_noalloc(f_dev.value, capi.STORAGE_NAMES[storage], lay["block_stride"],
                                                    lay["dir_stride"], obst.data_ptr(), case.dom.n_blocks,
                                                    out.data_ptr(), None))
    torch.cuda.synchronize()
    expect = L.mass_momentum()
    np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=RTOL, atol=1e-12 * abs(expect[0]))
    L.close()
    g.close()


def test_noalloc_periodic_without_obstacle(oal):
    import torch
    case = taylor_green_case(16, u0=0.05, re=100.0, c_wale=0.2)
    g = Geometry(case.dom)
    L = Level(g, storage="f32")
    L.init_equilibrium(case.rho, case.vel)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    for _ in range(2):
        L.perform_timestep(case.params)
        expect = L.mass_momentum()
        _noalloc(L, None, out, case.dom.n_blocks)
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=RTOL, atol=1e-12 * abs(expect[0]))
    L.close()
    g.close()


def test_noalloc_rejects_sizes_beyond_the_fixed_scratch(oal):
    import torch
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    st = capi.lib().oal_mass_momentum_noalloc(dummy.data_ptr(), capi.OAL_STORE_F32, 27 * 512, 512, None,
                                              capi.OAL_NOALLOC_MAX_BLOCKS + 1, out.data_ptr(), None)
    assert st == capi.OAL_E_TOO_LARGE
    assert b"exceeds" in capi.lib().oal_last_error()
