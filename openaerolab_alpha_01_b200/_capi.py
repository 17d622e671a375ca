"""ctypes bindings of liboal.so (declarations of include/oal.h).

The library is loaded from the package directory; a missing library raises immediately (there is
no CPU fallback on the product path).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
# OAL_LIBRARY selects another build of the library (for instance a tuning variant)
LIB_PATH = Path(os.environ.get("OAL_LIBRARY", str(PKG / "liboal.so")))

OAL_ABI_VERSION = 1

# status codes
OAL_OK = 0
OAL_E_INVALID_ARG = -1
OAL_E_UNKNOWN_OPERATOR = -2
OAL_E_CUDA = -3
OAL_E_OUT_OF_MEMORY = -4
OAL_E_UNSUPPORTED = -5
OAL_E_ABI_MISMATCH = -6
OAL_E_ADMISSION = -7
OAL_E_TOO_LARGE = -8
OAL_E_NOT_FOUND = -9
OAL_E_TIMEOUT = -10
OAL_E_NO_DEVICE = -11

OAL_OP_CUMULANT_D3Q27 = 1
OAL_OP_ENTROPIC_D3Q39 = 2
OAL_OP_HRR_D3Q19 = 3

OAL_STORE_F32 = 0
OAL_STORE_F16_DEV = 1
OAL_STORE_BF16_DEV = 2
OAL_STORE_F64 = 3

OAL_LIMITER_NONE = 0
OAL_LIMITER_FACTORED = 1
OAL_LIMITER_POSITIVITY = 2

OAL_LEVEL_DENSE = 1
OAL_LEVEL_ROUND_NEAREST = 2
OAL_LEVEL_EXACT_MATH = 4
OAL_TUNE_PREFETCH_CTAS = 1
OAL_TUNE_PERSISTENT = 2
OAL_TUNE_CANDIDATES = 8

OAL_SOLID_FULLWAY = 0
OAL_SOLID_HALFWAY = 1
OAL_SOLID_GRAD = 2
OAL_SOLID_BOUZIDI = 3

STORAGE_NAMES = {"f32": OAL_STORE_F32, "f16": OAL_STORE_F16_DEV, "bf16": OAL_STORE_BF16_DEV, "f64": OAL_STORE_F64}


class StepParams(C.Structure):
    """oal_step_params: scalar arguments of one level step (timestep.jl:1238-1478)."""

    _fields_ = [
        ("abi_version", C.c_uint32),
        ("operator_id", C.c_int32),
        ("tau", C.c_float),
        ("tau_parent", C.c_float),
        ("c_wale", C.c_float),
        ("nu_sgs_background", C.c_float),
        ("amr_sgs_scale", C.c_float),
        ("omega_bulk", C.c_float),
        ("omega3", C.c_float),
        ("omega4", C.c_float),
        ("adaptive_omega4", C.c_int32),
        ("lambda_param", C.c_float),
        ("limiter_type", C.c_int32),
        ("compressible_corr", C.c_int32),
        ("u_inlet", C.c_float),
        ("inlet_turbulence", C.c_float),
        ("time_step_seed", C.c_int32),
        ("ymin_wall_bc", C.c_int32),
        ("zwall_bc", C.c_int32),
        ("wall_model_active", C.c_int32),
        ("wall_model_max_distance", C.c_float),
        ("sponge_blend_distributions", C.c_int32),
        ("transverse_freestream", C.c_int32),
        ("transverse_freestream_blend", C.c_float),
        ("solid_bc", C.c_int32),
        ("collect_forces", C.c_int32),
        ("store_post_collision", C.c_int32),
        ("temporal_weight", C.c_float),
        ("use_temporal_interp", C.c_int32),
        ("level_visc_physical", C.c_int32),
        ("hrr_hybrid", C.c_int32),
        ("hrr_sigma", C.c_float),
        ("nu_sgs_lattice_floor", C.c_float),
        ("shock_nu_max", C.c_float),
        ("grad_pineq_scale", C.c_float),
        ("variable_nu_sgs", C.c_int32),
        ("c_pi", C.c_float),
        ("nu_sgs_floor", C.c_float),
        ("svv_x_epsilon", C.c_float),
        ("svv_yz_epsilon", C.c_float),
    ]


class SurfaceParams(C.Structure):
    """oal_surface_params (include/oal.h): the surface-stress mapping's settings."""
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("search_radius", C.c_int32),
        ("recover_normal", C.c_int32),
        ("tau", C.c_float),
        ("c_wale", C.c_float),
        ("nu_sgs_background", C.c_float),
        ("pressure_scale", C.c_float),
        ("stress_scale", C.c_float),
        ("moment_center", C.c_float * 3),
        ("reserved", C.c_int32 * 3),
    ]


class NscbcParams(C.Structure):
    """oal_nscbc_params (include/oal.h): the characteristic outlet's settings."""
    _fields_ = [
        ("enabled", C.c_int32),
        ("all_blocks", C.c_int32),
        ("p_target", C.c_float),
        ("sigma_relax", C.c_float),
        ("neq_blend", C.c_float),
        ("reserved", C.c_int32 * 3),
    ]


class GeometryDesc(C.Structure):
    _fields_ = [
        ("n_blocks", C.c_int32),
        ("nx_global", C.c_int32),
        ("ny_global", C.c_int32),
        ("nz_global", C.c_int32),
        ("active_coords", C.POINTER(C.c_int32)),
        ("neighbor_table", C.POINTER(C.c_int32)),
        ("obstacle", C.POINTER(C.c_uint8)),
        ("sponge", C.POINTER(C.c_float)),
        ("wall_dist", C.POINTER(C.c_float)),
    ]


class AmrLevelDesc(C.Structure):
    _fields_ = [
        ("geometry", C.c_void_p),
        ("dim", C.c_int32 * 3),
        ("reserved", C.c_int32),
    ]


class LevelFields(C.Structure):
    _fields_ = [
        ("f_in", C.c_void_p),
        ("f_out", C.c_void_p),
        ("f_post_collision", C.c_void_p),
        ("rho_out", C.c_void_p),
        ("vel_out", C.c_void_p),
        ("vel_in", C.c_void_p),
        ("storage", C.c_int32),
        ("reserved0", C.c_int32),
        ("f_block_stride", C.c_int64),
        ("f_dir_stride", C.c_int64),
        ("vel_comp_stride", C.c_int64),
        ("force_out", C.c_void_p),
    ]


OAL_Q19_SGS_NONE = 0
OAL_Q19_SGS_WALE = 1
OAL_Q19_SGS_SMAGORINSKY = 2
OAL_Q19_SGS_VREMAN = 3


class Q19Params(C.Structure):
    """oal_q19_params (include/oal.h): the octree level's numerics."""
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("sgs", C.c_int32),
        ("nu", C.c_double),
        ("c_wale", C.c_double),
        ("c_smagorinsky", C.c_double),
        ("hrr_sigma", C.c_double),
        ("body_force", C.c_double * 3),
        ("u_inlet", C.c_double * 3),
        ("force_scale", C.c_double),
    ]


OAL_Q19_K_NONE, OAL_Q19_K_FLUID, OAL_Q19_K_SOLID, OAL_Q19_K_COVERED, OAL_Q19_K_GHOST, OAL_Q19_K_BOUNDARY = range(6)
(OAL_Q19_FACE_PERIODIC, OAL_Q19_FACE_INLET, OAL_Q19_FACE_OUTLET, OAL_Q19_FACE_SLIP, OAL_Q19_FACE_SYMMETRY,
 OAL_Q19_FACE_NOSLIP, OAL_Q19_FACE_GROUND, OAL_Q19_FACE_FREESTREAM) = range(8)
Q19_FACE_NAMES = {"periodic": 0, "inlet": 1, "outlet": 2, "slip": 3, "symmetry": 4, "noslip": 5, "ground": 6,
                  "freestream": 7}


class Q19LevelDesc(C.Structure):
    """oal_q19_level_desc (include/oal.h): one octree level's arrays (the reference's OctLevel)."""
    _fields_ = [
        ("nocts", C.c_int32),
        ("origin", C.c_void_p),
        ("real", C.c_void_p),
        ("onbr", C.c_void_p),
        ("kind", C.c_void_p),
        ("face", C.c_void_p),
        ("special", C.c_void_p),
        ("cutidx", C.c_void_p),
        ("ncut", C.c_int32),
        ("cut_slot", C.c_void_p),
        ("cut_off", C.c_void_p),
        ("nlinks", C.c_int32),
        ("cut_dir", C.c_void_p),
        ("cut_q", C.c_void_p),
        ("cut_tri", C.c_void_p),
        ("cut_partner", C.c_void_p),
        ("ntri", C.c_int32),
        ("faces", C.c_int32 * 6),
        ("nghost", C.c_int32),
        ("ghost_slot", C.c_void_p),
        ("ghost_donor", C.c_void_p),
        ("ghost_w", C.c_void_p),
        ("nrestrict", C.c_int32),
        ("restrict_slot", C.c_void_p),
        ("restrict_src", C.c_void_p),
        ("restrict_cubic", C.c_void_p),
    ]


class Q19Region(C.Structure):
    """oal_q19_region (include/oal.h): a refinement region (0 box, 1 sphere, 2 cylinder)."""
    _fields_ = [
        ("kind", C.c_int32),
        ("level", C.c_int32),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("centre", C.c_double * 3),
        ("radius", C.c_double),
    ]


class Q19MeshSpec(C.Structure):
    """oal_q19_mesh_spec (include/oal.h): the reference's MeshSpec."""
    _fields_ = [
        ("domain", C.c_double * 3),
        ("dx", C.c_double),
        ("periodic", C.c_int32 * 3),
        ("faces", C.c_int32 * 6),
        ("levels", C.c_int32),
        ("surface_level", C.c_int32),
        ("band_fine", C.c_int32),
        ("band", C.c_int32),
        ("wake_level_offset", C.c_int32),
        ("wake_length", C.c_double),
        ("wake_margin", C.c_double),
        ("nregions", C.c_int32),
        ("regions", C.c_void_p),
        ("seal_cavities", C.c_int32),
        ("nsurface_levels", C.c_int32),
        ("surface_levels", C.c_void_p),
        ("reserved", C.c_int32 * 2),
    ]


class Q19SurfaceLevel(C.Structure):
    """oal_q19_surface_level (include/oal.h): SurfaceLevel of generator.jl:18-21."""
    _fields_ = [("level", C.c_int32), ("lo", C.c_double * 3), ("hi", C.c_double * 3)]


class OALError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"oal status {status}: {msg}")
        self.status = status


# Every symbol declared in include/oal.h, with its ctypes signature.
_SIGNATURES = {
    "oal_abi_version": (C.c_int32, []),
    "oal_status_string": (C.c_char_p, [C.c_int32]),
    "oal_last_error": (C.c_char_p, []),
    "oal_device_count": (C.c_int32, []),
    "oal_lookup_operator": (C.c_int32, [C.c_char_p, C.POINTER(C.c_int32)]),
    "oal_default_step_params": (None, [C.POINTER(StepParams)]),
    "oal_default_entropic_params": (None, [C.POINTER(StepParams)]),
    "oal_build_box_blocks": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32)]),
    "oal_build_sphere_obstacle": (C.c_int32, [C.c_int32, C.POINTER(C.c_int32), C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.POINTER(C.c_uint8), C.POINTER(C.c_int64)]),
    "oal_geometry_create": (C.c_int32, [C.POINTER(GeometryDesc), C.c_int32, C.POINTER(C.c_void_p)]),
    "oal_geometry_destroy": (None, [C.c_void_p]),
    "oal_geometry_info": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "oal_stream_collide": (C.c_int32, [C.c_void_p, C.POINTER(LevelFields), C.POINTER(StepParams), C.c_void_p]),
    "oal_level_create": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "oal_level_destroy": (None, [C.c_void_p]),
    "oal_level_create_ex": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_uint32, C.POINTER(C.c_void_p)]),
    "oal_level_init_equilibrium": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "oal_level_set_state": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_level_get_state": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_level_step": (C.c_int32, [C.c_void_p, C.POINTER(StepParams), C.c_void_p]),
    "oal_level_advance": (C.c_int32, [C.c_void_p, C.POINTER(StepParams), C.c_int32, C.c_void_p]),
    "oal_level_get_forces": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "oal_level_set_bouzidi": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint16),
                                          C.c_float, C.c_int32, C.c_float, C.c_float]),
    "oal_bouzidi_create": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint16),
                                       C.c_float, C.c_int32, C.c_float, C.c_float, C.POINTER(C.c_void_p)]),
    "oal_bouzidi_destroy": (None, [C.c_void_p]),
    "oal_bouzidi_apply": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_batch_set_bouzidi": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint16),
                                          C.c_float, C.c_int32, C.c_float, C.c_float]),
    "oal_level_get_forces_async": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_level_mass_momentum": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "oal_level_set_surface": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p]),
    "oal_default_surface_params": (None, [C.c_void_p]),
    "oal_level_surface_forces": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "oal_level_pi_neq": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "oal_default_nscbc_params": (None, [C.c_void_p]),
    "oal_level_set_nscbc": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "oal_level_set_tuning": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64]),
    "oal_level_get_tuning": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "oal_level_autotune": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_level_device_state": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                           C.POINTER(C.c_void_p)]),
    "oal_level_device_bytes": (C.c_int64, [C.c_void_p]),
    "oal_level_layout": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "oal_level_entropic_lambda": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_amr_create": (C.c_int32, [C.c_int32, C.POINTER(AmrLevelDesc), C.c_int32, C.POINTER(C.c_void_p)]),
    "oal_amr_destroy": (None, [C.c_void_p]),
    "oal_amr_level": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "oal_amr_advance": (C.c_int32, [C.c_void_p, C.POINTER(StepParams), C.c_int32, C.c_void_p]),
    "oal_batch_create": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                     C.POINTER(C.c_void_p)]),
    "oal_batch_destroy": (None, [C.c_void_p]),
    "oal_batch_add": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(StepParams), C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_int32)]),
    "oal_batch_remove": (C.c_int32, [C.c_void_p, C.c_int32]),
    "oal_batch_set_params": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(StepParams)]),
    "oal_batch_advance": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p]),
    "oal_batch_set_tuning": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64]),
    "oal_batch_get_tuning": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "oal_batch_autotune": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_batch_get_state": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_batch_get_forces": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "oal_batch_mass_momentum": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "oal_batch_info": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "oal_geometry_blocks": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "oal_mass_momentum_noalloc": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_int32,
                                              C.c_void_p, C.c_void_p]),
    "oal_q19_default_params": (C.c_int32, [C.POINTER(Q19Params)]),
    "oal_q19_periodic_box": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "oal_q19_level_create": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "oal_q19_level_destroy": (C.c_int32, [C.c_void_p]),
    "oal_q19_level_initialise": (C.c_int32, [C.c_void_p, C.POINTER(Q19Params), C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_level_advance": (C.c_int32, [C.c_void_p, C.POINTER(Q19Params), C.c_int32, C.c_int32, C.c_void_p]),
    "oal_q19_level_forces": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_level_create_desc": (C.c_int32, [C.c_int32, C.c_int32, C.POINTER(Q19LevelDesc), C.POINTER(C.c_void_p)]),
    "oal_q19_default_mesh_spec": (C.c_int32, [C.POINTER(Q19MeshSpec)]),
    "oal_q19_mesh_generate": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(Q19MeshSpec), C.POINTER(C.c_void_p)]),
    "oal_q19_mesh_destroy": (C.c_int32, [C.c_void_p]),
    "oal_q19_mesh_counts": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "oal_q19_mesh_seal_counts": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64)]),
    "oal_q19_mesh_level_desc": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(Q19LevelDesc)]),
    "oal_q19_mesh_levels": (C.c_int32, [C.c_void_p]),
    "oal_q19_octree_create": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "oal_q19_octree_destroy": (C.c_int32, [C.c_void_p]),
    "oal_q19_octree_level": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "oal_q19_octree_initialise": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_octree_advance": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "oal_q19_octree_forces": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_octree_totals": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "oal_q19_level_get_state": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_level_set_state": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_level_get_buffer": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_level_set_buffer": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oal_q19_level_device_state": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                               C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    "oal_q19_level_totals": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "oal_q19_collide_cells": (C.c_int32, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}

OAL_NOALLOC_MAX_BLOCKS = 65536

_lib = None


def lib() -> C.CDLL:
    """Load liboal.so once (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m openaerolab_alpha_01_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.oal_abi_version() != OAL_ABI_VERSION:
            raise RuntimeError("liboal ABI version mismatch")
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OAL_OK:
        msg = lib().oal_last_error().decode(errors="replace")
        raise OALError(status, msg)


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def default_params(**overrides) -> StepParams:
    p = StepParams()
    lib().oal_default_step_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p
