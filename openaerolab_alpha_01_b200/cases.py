"""Case builders for the standard workloads: the periodic Taylor-Green box and the sphere channel.

* ``taylor_green_case`` — uniform n^3 fully periodic box (every neighbour-table entry wraps, which
  turns the reference's level kernel into a periodic one), 2-D Taylor-Green vortex uniform in z,
  Re from u0 L / nu with L = n / (2 pi).
* ``entropic_taylor_green_case`` — the same periodic box for the D3Q39 entropic KBC level
  (cs^2 = 2/3, so tau = nu / cs^2 + 1/2), FP32.
* ``sphere_channel_case`` — nx x ny x nz channel, velocity inlet at x_min
  (src/collision/kernel_cumulant.jl:235-239), zero-gradient outlet (:240-245), lateral mirrors
  (:342-345), analytic sphere (src/geometry/domain_generation.jl:132-150) with half-way
  bounce-back and the FP64 momentum-exchange drag.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from .solver import BlockDomain, apply_analytic_sphere_obstacle, build_box, taylor_green_fields


@dataclass
class Case:
    name: str
    dom: BlockDomain
    rho: np.ndarray
    vel: np.ndarray
    params: capi.StepParams
    meta: dict = field(default_factory=dict)

    @property
    def fluid_cells(self) -> int:
        n = self.dom.n_blocks * 512
        if self.dom.obstacle is not None:
            n -= int(np.count_nonzero(self.dom.obstacle))
        return n


def taylor_green_case(n: int, u0: float = 0.05, re: float = 100.0, c_wale: float = 0.0,
                      phase: tuple[float, float] = (0.0, 0.0), **overrides) -> Case:
    if n % 8:
        raise ValueError("box edge must be a multiple of 8")
    dom = build_box(n // 8, n // 8, n // 8, periodic=(True, True, True))
    L = n / (2.0 * np.pi)
    nu = u0 * L / re
    tau = 3.0 * nu + 0.5
    rho, vel = taylor_green_fields(dom, u0, phase)
    p = capi.default_params(tau=tau, c_wale=c_wale, u_inlet=0.0, **overrides)
    return Case(f"tgv{n}", dom, rho, vel, p, dict(u0=u0, re=re, nu=nu, tau=tau, k=2 * np.pi / n))


def entropic_taylor_green_case(n: int, u0: float = 0.1, re: float = 1000.0, c_wale: float = 0.2,
                               **overrides) -> Case:
    if n % 8:
        raise ValueError("box edge must be a multiple of 8")
    from .solver import default_entropic_params
    dom = build_box(n // 8, n // 8, n // 8, periodic=(True, True, True))
    L = n / (2.0 * np.pi)
    nu = u0 * L / re
    tau = nu / (2.0 / 3.0) + 0.5
    rho, vel = taylor_green_fields(dom, u0)
    p = default_entropic_params(tau=tau, c_wale=c_wale, u_inlet=0.0, **overrides)
    return Case(f"kbc_tgv{n}", dom, rho, vel, p, dict(u0=u0, re=re, nu=nu, tau=tau, k=2 * np.pi / n))


def sphere_channel_case(nx: int = 256, ny: int = 128, nz: int = 128, diameter: float = 24.0,
                        centre_x: float = 64.0, u_inlet: float = 0.05, re: float = 1000.0,
                        c_wale: float = 0.20, solid_bc: int = capi.OAL_SOLID_HALFWAY, **overrides) -> Case:
    if nx % 8 or ny % 8 or nz % 8:
        raise ValueError("channel sizes must be multiples of 8")
    dom = build_box(nx // 8, ny // 8, nz // 8)
    centre = (centre_x, ny / 2.0, nz / 2.0)
    n_solid = apply_analytic_sphere_obstacle(dom, centre, diameter / 2.0)
    nu = u_inlet * diameter / re
    tau = 3.0 * nu + 0.5
    nb = dom.n_blocks
    rho = np.ones((nb, 512))
    vel = np.zeros((3, nb, 512))
    vel[0] = np.where(dom.obstacle != 0, 0.0, u_inlet)
    p = capi.default_params(tau=tau, c_wale=c_wale, u_inlet=u_inlet, solid_bc=solid_bc, collect_forces=1, **overrides)
    area = np.pi * diameter * diameter / 4.0
    return Case(f"sphere_channel_{nx}x{ny}x{nz}", dom, rho, vel, p,
                dict(nu=nu, tau=tau, re=re, diameter=diameter, centre=centre, n_solid=n_solid,
                     drag_scale=1.0 / (0.5 * u_inlet * u_inlet * area)))
