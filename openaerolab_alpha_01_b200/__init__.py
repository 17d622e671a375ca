"""B200-native (sm_100a) lattice-Boltzmann level step behind the OpenAeroLab solver-step API.

The compute path is liboal.so (hand-written CUDA, C ABI in include/oal.h); this package holds
its ctypes bindings and the host-side mirror of the reference's operator and step interface.
"""
from ._capi import OALError, lib, default_params, StepParams  # noqa: F401
from .solver import (  # noqa: F401
    Batch,
    BlockDomain,
    Geometry,
    Level,
    apply_analytic_sphere_obstacle,
    build_box,
    default_step_params,
    get_collision_kernel,
    kinetic_energy,
    taylor_green_fields,
)

__all__ = [
    "OALError", "lib", "default_params", "StepParams", "Batch", "BlockDomain", "Geometry", "Level",
    "apply_analytic_sphere_obstacle", "build_box", "default_step_params", "get_collision_kernel",
    "kinetic_energy", "taylor_green_fields",
]
