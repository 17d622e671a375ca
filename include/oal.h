/*
 * oal.h — C ABI of liboal, the B200 (sm_100a) lattice-Boltzmann step library.
 *
 * The entry points below are what a Julia `ccall` shim binds in place of the reference's
 * solver-step and collision-operator API (OpenAeroLab, Julia + KernelAbstractions):
 *
 *   reference                                              replaced by
 *   -----------------------------------------------------  ------------------------------------
 *   get_collision_kernel(op, backend, is_l1)               oal_lookup_operator
 *     src/collision/physics_kernels.jl:50-75
 *   scalar kernel args `_kargs` + isbits param packs       oal_step_params / oal_default_step_params
 *     src/collision/timestep.jl:1238-1478,
 *     src/collision/kernel_param_packs.jl:45-76,
 *     defaults src/io/config_loader.jl:1305-1380
 *   build_neighbor_table(active_coords, bx,by,bz)          oal_build_box_blocks
 *     src/geometry/domain_topology.jl:919-953
 *   apply_analytic_sphere_obstacle!                        oal_build_sphere_obstacle
 *     src/geometry/domain_generation.jl:111-154
 *   BlockLevel arrays (f, f_temp, rho, vel, obstacle ...)  oal_geometry_* + oal_level_*
 *     src/geometry/blocks.jl:14-364
 *   stream_collide_cumulant!(f_out, f_in, ..., ndrange)    oal_stream_collide (caller-owned arrays)
 *     src/collision/kernel_cumulant.jl:29-912              oal_level_step   (library-owned arrays)
 *   stream_collide_entropic_d3q39!(...) + lambda_cache     oal_level_step with OAL_OP_ENTROPIC_D3Q39
 *     src/collision/kernel_entropic_d3q39.jl:529-3368,     oal_level_entropic_lambda
 *     timestep.jl:1133-1143,1447-1450                      oal_default_entropic_params
 *   perform_timestep_v2!(level, ...) launch + ping-pong    oal_level_step / oal_level_advance
 *     src/collision/timestep.jl:946-1559,
 *     src/solver/solver_control.jl:85-119
 *   init kernels (equilibrium start)                       oal_level_init_equilibrium
 *     src/main.jl:546-600
 *   total mass / momentum (Float64)                        oal_level_mass_momentum
 *     src/octree_q19/src/state.jl:614-637
 *   momentum-exchange force (Float64 per cut link)         oal_level_get_forces
 *     src/octree_q19/src/stream.jl:248-256,382-389
 *
 * Conventions
 *   - Every function returns OAL_OK (0) or a negative oal_status; oal_last_error() gives the
 *     text of the last failure on the calling host thread.
 *   - Arrays named "host" are plain host memory; arrays named "device" are CUDA device pointers.
 *   - Array layouts follow the reference (Julia, column-major, 1-based indices):
 *       populations  f(8,8,8,n_blocks,Q)       element (x,y,z,b,k) at x + 8y + 64z + 512b + 512*n_blocks*k
 *       density      rho(8,8,8,n_blocks)
 *       velocity     vel(8,8,8,n_blocks,3)
 *       obstacle     obstacle(8,8,8,n_blocks)   (Bool / uint8, nonzero = solid)
 *       neighbours   neighbor_table(n_blocks,27) 1-based block index, 0 = none,
 *                    direction (dx,dy,dz) at (dx+1) + 3(dy+1) + 9(dz+1)   (0-based column)
 *       block coords active_coords (bx,by,bz) 1-based, stored as n_blocks rows of 3
 *   - Streams are passed as `void*` (a cudaStream_t; NULL = the legacy default stream).
 *   - A context object (geometry, level, batch, server) is not thread-safe: one host thread
 *     drives it at a time. Different objects may be driven from different threads.
 */
#ifndef OAL_H
#define OAL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OAL_ABI_VERSION 1

typedef int32_t oal_status;
enum {
  OAL_OK = 0,
  OAL_E_INVALID_ARG = -1,
  OAL_E_UNKNOWN_OPERATOR = -2, /* physics_kernels.jl:71-74 error() */
  OAL_E_CUDA = -3,
  OAL_E_OUT_OF_MEMORY = -4,
  OAL_E_UNSUPPORTED = -5,
  OAL_E_ABI_MISMATCH = -6,
  OAL_E_ADMISSION = -7, /* request does not fit the HBM budget */
  OAL_E_TOO_LARGE = -8,
  OAL_E_NOT_FOUND = -9,
  OAL_E_TIMEOUT = -10,
  OAL_E_NO_DEVICE = -11
};

/* Collision operators (reference symbols :cumulant, :entropic, octree :hrr). */
enum {
  OAL_OP_CUMULANT_D3Q27 = 1,
  OAL_OP_ENTROPIC_D3Q39 = 2,
  OAL_OP_HRR_D3Q19 = 3
};

/* Population storage codecs. DEV = deviation (f/w_k - 1) from the lattice weight. */
enum {
  OAL_STORE_F32 = 0,
  OAL_STORE_F16_DEV = 1,
  OAL_STORE_BF16_DEV = 2,
  OAL_STORE_F64 = 3
};

/* Cumulant limiter codes (config_loader.jl:1378-1383, timestep.jl:1158-1163). */
enum { OAL_LIMITER_NONE = 0, OAL_LIMITER_FACTORED = 1, OAL_LIMITER_POSITIVITY = 2 };

/* Treatment of solid (obstacle) cells.
 *   FULLWAY: the reference's "simple bounce-back" inside obstacle cells
 *            (kernel_cumulant.jl:402-417); fluid cells pull from solid cells unchanged.
 *   HALFWAY: half-way bounce-back on every fluid->solid link with the momentum-exchange
 *            force of the octree solver (octree_q19/src/stream.jl:229-256) on D3Q27 links;
 *            solid cells hold the rest equilibrium.
 *   GRAD:    FULLWAY, then the Grad-reconstruction wall of the reference's bc_scheme "grad"
 *            (geometry/grad_wall_kernel.jl:42-144, called from timestep.jl:1738-1751) on every
 *            fluid cell with a link into a solid cell: all its post-collision populations are
 *            rebuilt as f_eq(rho, u_wall = 0) + (1 - 1/tau) w_k 4.5 Q_k : Pi_neq (Pi_neq of the
 *            post-collision populations about (rho, 0), times grad_pineq_scale), floored at
 *            1e-12, and its velocity output set to 0 (wall velocity mode "none", the default).
 *            No momentum-exchange force is accumulated (forces come from HALFWAY).
 *   BOUZIDI: FULLWAY, then the linear Bouzidi correction of the reference's default bc_scheme
 *            "bouzidi_linear" (geometry/bouzidi_kernel.jl:150-380, called from timestep.jl:1752-1768)
 *            on the boundary cells and q values attached by oal_level_set_bouzidi; no attached
 *            cells = FULLWAY. No momentum-exchange force is accumulated. */
enum { OAL_SOLID_FULLWAY = 0, OAL_SOLID_HALFWAY = 1, OAL_SOLID_GRAD = 2, OAL_SOLID_BOUZIDI = 3 };

/* Scalar step parameters: the scalars of `_kargs` (timestep.jl:1238-1478) that the
 * D3Q27 level-1 path reads. Field meaning and units are the reference's (lattice units). */
typedef struct oal_step_params {
  uint32_t abi_version;          /* must be OAL_ABI_VERSION */
  int32_t operator_id;           /* OAL_OP_* */
  float tau;                     /* tau_molecular */
  float tau_parent;              /* parent level tau (refined levels) */
  float c_wale;                  /* WALE constant (config default 0.20) */
  float nu_sgs_background;       /* background eddy viscosity (default 0) */
  float amr_sgs_scale;           /* SGS scale of the level (timestep.jl:1127: 1.0) */
  float omega_bulk;              /* default 1 */
  float omega3;                  /* default 1 */
  float omega4;                  /* default 1 */
  int32_t adaptive_omega4;       /* default 1 */
  float lambda_param;            /* default 1/6 */
  int32_t limiter_type;          /* OAL_LIMITER_*, default FACTORED */
  int32_t compressible_corr;     /* 1 = O(u^4) Hermite equilibrium, default 0 */
  float u_inlet;                 /* inlet velocity (x) */
  float inlet_turbulence;        /* inlet noise amplitude (fraction of u_inlet) */
  int32_t time_step_seed;        /* noise seed (the step counter) */
  int32_t ymin_wall_bc;          /* 1 = bounce-back ground at y_min */
  int32_t zwall_bc;              /* 0 legacy mirror, 1 slip, 2 no-slip */
  int32_t wall_model_active;     /* Werner-Wengle / log-law wall model */
  float wall_model_max_distance; /* cells */
  int32_t sponge_blend_distributions;
  int32_t transverse_freestream;
  float transverse_freestream_blend;
  int32_t solid_bc;              /* OAL_SOLID_* */
  int32_t collect_forces;        /* accumulate the FP64 momentum-exchange force this step */
  int32_t store_post_collision;  /* also write f_post_collision */
  float temporal_weight;         /* refined levels (reserved) */
  int32_t use_temporal_interp;   /* refined levels (reserved) */
  int32_t level_visc_physical;   /* refined levels (reserved) */
  /* D3Q39 entropic operator only (kernel_entropic_d3q39.jl arguments of the same names); for that
   * operator `lambda_param` is the h-damping sigma (timestep.jl:1142) and `adaptive_omega4` the
   * alpha solver: 0 bisection, 1 Newton, 2 approximate, 3 Taylor (timestep.jl:1139-1141). */
  int32_t hrr_hybrid;            /* 1 = HRR-hybrid stress reconstruction (default 0) */
  float hrr_sigma;               /* HRR blend, used when hrr_hybrid and < 0.999 (default 1) */
  float nu_sgs_lattice_floor;    /* level-independent lattice-viscosity floor (default 0) */
  float shock_nu_max;            /* Mach-pocket viscosity: max(5 shock_nu_max, 0.24) (default 0) */
  /* OAL_SOLID_GRAD: share of Pi_neq the wall keeps (config grad_pineq_scale, default 1) */
  float grad_pineq_scale;
  /* Variable eddy viscosity of the D3Q27 step (kernel_cumulant.jl:546-588): 0 = WALE with the
   * background floor (VARIABLE_NU_SGS false, the default); 1 = nu_sgs from the previous step's
   * post-collision Pi_neq, c_pi |Pi_pre| / (rho cs^2) (VARIABLE_NU_SGS); 2 = the Germano-Lilly
   * dynamic coefficient from a 7-point test filter of the velocity (kernel_dynamic_sgs.jl,
   * DYNAMIC_SGS_ENABLED). Modes 1 and 2 floor nu_sgs at nu_sgs_floor and cap it at 0.1; every
   * block of the level then steps in the general kernel. Library-owned levels only. */
  int32_t variable_nu_sgs;
  float c_pi;                    /* VARIABLE_NU_SGS_C_PI (default 0.2) */
  float nu_sgs_floor;            /* VARIABLE_NU_SGS_FLOOR (default 0.002) */
  /* Spectral vanishing viscosity (kernel_svv_yz_d3q39.jl): the strength of the 5-point bi-Laplacian
   * filter along x and along y and z on this level, 0 = off (the default). The reference applies
   * SVV_X_EPSILON on levels <= SVV_X_MAX_LEVEL and SVV_YZ_EPSILON on levels >= SVV_YZ_MIN_LEVEL
   * (1-based, timestep.jl:1577-1578); the caller passes the level's values. D3Q27: a post-pass after
   * the step kernels, before the outlet and the wall corrections (timestep.jl:1576-1611); D3Q39:
   * inside the step, after the post-collision guard (kernel_entropic_d3q39.jl:3256-3310). On
   * caller-owned arrays (oal_stream_collide) the filter also writes f_post_collision when given;
   * batched cases refuse a non-zero strength. */
  float svv_x_epsilon;
  float svv_yz_epsilon;
} oal_step_params;

/* ---- library ---------------------------------------------------------------------------- */
int32_t oal_abi_version(void);
const char* oal_status_string(oal_status s);
const char* oal_last_error(void);
/* Number of CUDA devices visible (0 when none). */
int32_t oal_device_count(void);

/* Operator registry: "cumulant" -> OAL_OP_CUMULANT_D3Q27, "entropic" -> OAL_OP_ENTROPIC_D3Q39,
 * "hrr"/"octree_q19" -> OAL_OP_HRR_D3Q19; anything else -> OAL_E_UNKNOWN_OPERATOR.
 * Replaces get_collision_kernel (src/collision/physics_kernels.jl:50-75). */
oal_status oal_lookup_operator(const char* name, int32_t* out_operator_id);

/* Fill `p` with the reference's configuration defaults (src/io/config_loader.jl:1305-1380). */
void oal_default_step_params(oal_step_params* p);
/* The same with the D3Q39 entropic operator selected and its slots set as timestep.jl:1133-1143
 * sets them: lambda_param = ENTROPIC_SIGMA (0), adaptive_omega4 = alpha solver (0, bisection). */
void oal_default_entropic_params(oal_step_params* p);

/* ---- host-side domain builders ------------------------------------------------------------ */
/* Active blocks of a full bx_max x by_max x bz_max box in the reference's sorted order
 * (tuples sorted lexicographically, src/geometry/domain.jl:785) and their 27-entry
 * neighbour table (domain_topology.jl:919-953). periodic_mask bit 0/1/2 wraps x/y/z.
 * coords_out: host int32[n*3] (n = bx_max*by_max*bz_max); nbr_out: host int32[n*27],
 * Julia column-major (n,27). */
oal_status oal_build_box_blocks(int32_t bx_max, int32_t by_max, int32_t bz_max,
                                int32_t periodic_mask, int32_t* coords_out, int32_t* nbr_out);

/* Analytic sphere mask (domain_generation.jl:132-150): cell (lx,ly,lz) of block (bx,by,bz) is
 * solid when its centre ((b-1)*8 + l - 0.5, cell units) lies within `radius` of `centre`.
 * obstacle_out: host uint8[512*n_blocks]. Returns the solid count in *n_solid (may be NULL). */
oal_status oal_build_sphere_obstacle(int32_t n_blocks, const int32_t* coords,
                                     double cx, double cy, double cz, double radius,
                                     uint8_t* obstacle_out, int64_t* n_solid);

/* ---- geometry (device-resident topology of one level) -------------------------------------- */
typedef struct oal_geometry_desc {
  int32_t n_blocks;
  int32_t nx_global, ny_global, nz_global; /* domain size in cells (boundary classification) */
  const int32_t* active_coords;            /* host int32[n_blocks*3] */
  const int32_t* neighbor_table;           /* host int32[n_blocks*27], Julia layout */
  const uint8_t* obstacle;                 /* host uint8[512*n_blocks] or NULL (all fluid) */
  const float* sponge;                     /* host float[512*n_blocks] or NULL */
  const float* wall_dist;                  /* host float[512*n_blocks] or NULL */
} oal_geometry_desc;

typedef struct oal_geometry oal_geometry;
oal_status oal_geometry_create(const oal_geometry_desc* desc, int32_t device, oal_geometry** out);
void oal_geometry_destroy(oal_geometry* g);
/* Counts: out[0]=n_blocks, out[1]=fluid cells, out[2]=solid cells, out[3]=boundary blocks,
 * out[4]=blocks needing per-cell solid masks. */
oal_status oal_geometry_info(const oal_geometry* g, int64_t out[5]);

/* ---- caller-owned arrays: drop-in for stream_collide_cumulant! ------------------------------ */
/* Device pointers of one level step, in the reference layout by default. Element strides let
 * the caller pass the library's block-major layout too. */
typedef struct oal_level_fields {
  const void* f_in;        /* device, storage type */
  void* f_out;             /* device, storage type */
  void* f_post_collision;  /* device or NULL */
  void* rho_out;           /* device float (double for OAL_STORE_F64) */
  void* vel_out;           /* device float/double */
  const void* vel_in;      /* device float/double (previous step's velocity) */
  int32_t storage;         /* OAL_STORE_* */
  int32_t reserved0;
  int64_t f_block_stride;  /* elements between blocks   (reference: 512) */
  int64_t f_dir_stride;    /* elements between directions (reference: 512*n_blocks) */
  int64_t vel_comp_stride; /* elements between velocity components (reference: 512*n_blocks) */
  double* force_out;       /* device double[3] receiving the momentum-exchange force, or NULL */
} oal_level_fields;

/* One fused pull-stream-collide step of a level-1 (no parent) D3Q27 cumulant level.
 * Stream-ordered, asynchronous; force_out (when collect_forces) is written by a second
 * stream-ordered reduction. Replaces stream_collide_cumulant! (kernel_cumulant.jl:29-912). */
oal_status oal_stream_collide(const oal_geometry* g, const oal_level_fields* fields,
                              const oal_step_params* p, void* stream);

/* ---- library-owned level state ---------------------------------------------------------- */
typedef struct oal_level oal_level;
/* operator_id OAL_OP_CUMULANT_D3Q27 (any storage) or OAL_OP_ENTROPIC_D3Q39 (OAL_STORE_F32; the
 * level's population arrays then have Q = 39 and step with oal_default_entropic_params). */
oal_status oal_level_create(const oal_geometry* g, int32_t operator_id, int32_t storage,
                            oal_level** out);
void oal_level_destroy(oal_level* L);
/* Level creation options (bits of `flags`). */
enum {
  OAL_LEVEL_DENSE = 1,         /* box levels in FP32/FP16/BF16: dense padded population grid */
  OAL_LEVEL_ROUND_NEAREST = 2, /* FP16/BF16 deviation storage: the step kernels round the stored
                                  deviations to nearest. Default: stochastic rounding (hardware
                                  cvt.rs, random bits hashed from the cell's position in its case
                                  and its new macros), unbiased in expectation, which keeps
                                  integrated quantities such as the drag free of the rounding bias
                                  of a slowly varying state. No counterpart in the reference (its
                                  populations are Float32). */
  OAL_LEVEL_EXACT_MATH = 4     /* D3Q39 entropic levels: exp and log by the software routines the
                                  CPU restatement shares (the step is then bit-identical to it).
                                  Default: CUDA's expf / logf, the functions the reference's
                                  Float32 exp and log compile to on its CUDA backend. */
};
/* oal_level_create with options; flags = 0 is oal_level_create. */
oal_status oal_level_create_ex(const oal_geometry* g, int32_t operator_id, int32_t storage, uint32_t flags,
                               oal_level** out);
/* Equilibrium start from host rho(8,8,8,nb) and vel(8,8,8,nb,3) in double precision:
 * f_k = feq(rho,u) (physics_utils.jl:30-35), vel_in = u. */
oal_status oal_level_init_equilibrium(oal_level* L, const double* rho_host, const double* vel_host,
                                      int32_t compressible_corr);
/* Overwrite the state from host arrays (reference layout, double precision). vel/rho may be NULL. */
oal_status oal_level_set_state(oal_level* L, const double* f_host, const double* rho_host,
                               const double* vel_host);
/* Read the current state (after the last step) into host arrays (reference layout, double).
 * Any pointer may be NULL. Synchronises the level's stream. */
oal_status oal_level_get_state(oal_level* L, double* f_host, double* rho_host, double* vel_host);
/* One step (ping-pong by parity, solver_control.jl:85-91). */
oal_status oal_level_step(oal_level* L, const oal_step_params* p, void* stream);
/* n steps as one captured CUDA graph (re-captured when n or p change); time_step_seed advances
 * by one per step inside the graph. */
oal_status oal_level_advance(oal_level* L, const oal_step_params* p, int32_t n_steps, void* stream);
/* Momentum-exchange force of the last step that collected it (lattice units, FP64).
 * Synchronises the level's stream. */
oal_status oal_level_get_forces(oal_level* L, double out[3]);

/* Boundary cells and link fractions of the linear Bouzidi wall (OAL_SOLID_BOUZIDI). Replaces
 * the per-level BouzidiDataSparse of the reference (geometry/bouzidi_common.jl:15-23, built by
 * compute_bouzidi_qmap_sparse, geometry/bouzidi_setup.jl:175-390) and the scalars that
 * apply_bouzidi_correction! takes (geometry/bouzidi_kernel.jl:382-432).
 *   cell_block, cell_x, cell_y, cell_z: n_cells 1-based entries (block of the level, x, y, z in
 *     1..8), the reference's bouzidi_cell_* arrays;
 *   q_half: n_cells x 27 IEEE binary16 link fractions, direction fastest in the D3Q27 order of
 *     the level (q_map[x, y, z, b, k] of each listed cell); a link is corrected when
 *     q_min_threshold < q <= 1;
 *   ff_fallback: 0 halfway_bb (default), 1 wall_eq, 2 bounce_back (config ff_fallback);
 *   limiter_rel_cap, limiter_abs_cap: wall_pop_limiter_rel_cap / _abs_cap (0 = off).
 * After every step of L with solid_bc OAL_SOLID_BOUZIDI, for each listed cell x and link k:
 * f_out[x, opp k] = 2q f*_k(x) + (1-2q) f*_k(x - c_k) if q < 1/2 (the fall-back when x - c_k is
 * solid or absent), else f*_k(x)/(2q) + (2q-1)/(2q) f*_opp k(x), f* the step's post-collision
 * populations. n_cells = 0 detaches. D3Q27 levels, on their own or of a hierarchy (oal_amr_level:
 * the correction follows each step of that level, before the restriction onto its parent); not
 * entropic levels, not batched cases. Copies the arrays; invalidates the captured step graphs. */
oal_status oal_level_set_bouzidi(oal_level* L, int32_t n_cells, const int32_t* cell_block, const int32_t* cell_x,
                                 const int32_t* cell_y, const int32_t* cell_z, const uint16_t* q_half,
                                 float q_min_threshold, int32_t ff_fallback, float limiter_rel_cap,
                                 float limiter_abs_cap);
/* Non-blocking variant: enqueue the copy of the force into a host buffer (pinned for overlap). */
oal_status oal_level_get_forces_async(oal_level* L, double* host_out3, void* stream);
/* Surface-stress force mapping of a D3Q27 or D3Q39 level (CS2_PHYSICS 1/3 or 2/3): the reference's compute_aerodynamics!
 * (src/forces/surface.jl:1577-1587) with its default Prandtl force method, i.e.
 * map_stresses_kernel! (:636-1031) over the triangles, compute_stress_from_cell (:180-269) and
 * integrate_forces_kernel! (:1265-1331). Triangles: centroid, unit outward normal and area per
 * row (tri[n * 7], cell units: cell (i, j, k), 1-based, is centred at (i - 1/2, j - 1/2, k - 1/2);
 * the reference's mesh_offset and dx folded in by the caller). oal_level_set_surface copies them
 * (n_tri = 0 detaches). */
oal_status oal_level_set_surface(oal_level* L, int32_t n_tri, const float* tri);
typedef struct oal_surface_params {
  uint32_t abi_version;     /* OAL_ABI_VERSION */
  int32_t search_radius;    /* probe steps along the normal (reference default 8) */
  int32_t recover_normal;   /* 1: closed bodies may take the opposite side (reference default) */
  float tau;                /* molecular relaxation time of the level */
  float c_wale;             /* C_SMAGO (config c_wale, default 0.20) */
  float nu_sgs_background;  /* NU_SGS_BACKGROUND (default 0) */
  float pressure_scale;     /* rho_phys u_scale^2 (1: lattice units) */
  float stress_scale;       /* the same for the shear (the reference uses pressure_scale) */
  float moment_center[3];   /* moment reference point (cell units) */
  int32_t reserved[3];
} oal_surface_params;
/* Fills `sp` with the reference's defaults. */
void oal_default_surface_params(oal_surface_params* sp);
/* Maps the stresses on the attached triangles from the level's current density and velocity.
 * out[9] = pressure force, viscous force, moment about moment_center (FP64, summed in a fixed
 * order; the reference adds Float32 atomics). per_tri (optional, host float[n * 6]): pressure,
 * shear x, y, z, normal sign (-1 where the opposite side was taken), probe wall distance (0: no
 * fluid found). Synchronous. */
oal_status oal_level_surface_forces(oal_level* L, const oal_surface_params* sp, double out[9], float* per_tri);

/* FP64 on-device reduction of the current state: out = {mass, px, py, pz} over fluid cells. */
oal_status oal_level_mass_momentum(oal_level* L, double out[4]);
/* Non-equilibrium stress of the current state (compute_pi_neq_kernel!, kernel_pi_neq.jl:39-180,
 * D3Q27): Pi_ab = sum_k c_a c_b (f_k - f_eq_k(rho, u)) at every cell, 0 in solid or unphysical
 * cells; host float out[6][n_blocks * 512] in the order xx, yy, zz, xy, xz, yz. */
oal_status oal_level_pi_neq(oal_level* L, float* out);
/* ---- linear Bouzidi walls on caller-owned arrays ------------------------------------------- */
/* apply_bouzidi_correction! (bouzidi_kernel.jl:150-380) as its own call, as perform_timestep_v2!
 * makes it after the kernel (timestep.jl:1752-1768): a set of boundary cells of a geometry
 * (arguments as oal_level_set_bouzidi), applied to the populations of a step that ran through
 * oal_stream_collide with solid_bc OAL_SOLID_BOUZIDI (full-way in the step); it reads and
 * corrects fl->f_out in the caller's layout. */
typedef struct oal_bouzidi oal_bouzidi;
oal_status oal_bouzidi_create(const oal_geometry* g, int32_t storage, int32_t n_cells, const int32_t* cell_block,
                              const int32_t* cell_x, const int32_t* cell_y, const int32_t* cell_z,
                              const uint16_t* q_half, float q_min_threshold, int32_t ff_fallback,
                              float limiter_rel_cap, float limiter_abs_cap, oal_bouzidi** out);
void oal_bouzidi_destroy(oal_bouzidi* bz);
oal_status oal_bouzidi_apply(const oal_geometry* g, oal_bouzidi* bz, const oal_level_fields* fl, void* stream);

/* ---- characteristic outlet (NSCBC, kernel_nscbc_outlet.jl) ---------------------------------- */
/* Poinsot-Lele outflow on the +x outlet plane (apply_nscbc_outlet_kernel!, :80-340), applied
 * after every step of a library-owned D3Q27 level: LODI relaxation of the incoming acoustic
 * characteristic toward p_target for subsonic outflow, capped Euler update of the face
 * macros (tangential characteristics dropped at lateral-wall corners), face populations rebuilt
 * as the equilibrium of the new state plus neq_blend times the interior cell's non-equilibrium
 * part. Athermal (T = 1, p = rho cs^2). Off by default. */
typedef struct oal_nscbc_params {
  int32_t enabled;      /* OUTLET_NSCBC_ENABLED (false) */
  int32_t all_blocks;   /* 0: the x = 8 plane of the blocks on the +x face; 1: of every block, the
                           range apply_nscbc_outlet! launches (its kernel checks no block coordinate) */
  float p_target;       /* OUTLET_NSCBC_P_TARGET (1.0) */
  float sigma_relax;    /* OUTLET_NSCBC_SIGMA (0.27) */
  float neq_blend;      /* OUTLET_NSCBC_NEQ_BLEND (0.5) */
  int32_t reserved[3];
} oal_nscbc_params;
void oal_default_nscbc_params(oal_nscbc_params* np);
oal_status oal_level_set_nscbc(oal_level* L, const oal_nscbc_params* np);

/* ---- launch tuning (no counterpart in the reference; results do not depend on it) ---------- */
/* OAL_TUNE_PREFETCH_CTAS: the x-pair kernel's CTA j also bulk-prefetches into L2 the populations
 * and velocities of the CTA prefetch_ctas launches ahead in its launch (0 = off, the default).
 * OAL_TUNE_PERSISTENT: 1 launches the x-pair kernel in its persistent form, as many CTAs as stay
 * resident walking the launch's units (0 = one CTA per unit, the default). */
#define OAL_TUNE_PREFETCH_CTAS 1
#define OAL_TUNE_PERSISTENT 2
#define OAL_TUNE_CANDIDATES 8
oal_status oal_level_set_tuning(oal_level* L, int32_t key, int64_t value);
oal_status oal_level_get_tuning(const oal_level* L, int32_t key, int64_t* value);
/* The autotuner: times n_steps steps (CUDA events, after one untimed run of the same n_steps) for
 * each of the OAL_TUNE_CANDIDATES settings (plain and persistent launch x prefetch distances
 * {0, 4, 8, 16} x the SM count), each from the level's current state, which is restored
 * afterwards (the level ends where it started), and keeps the fastest. prefetch[c],
 * persistent[c] and ms_per_step[c] (host, nullable) report every candidate. Needs device memory
 * for one copy of the state. */
oal_status oal_level_autotune(oal_level* L, const oal_step_params* p, int32_t n_steps, int64_t* prefetch,
                              int32_t* persistent, double* ms_per_step);
/* Device pointers of the current state (for zero-copy interop): f, rho, vel. */
oal_status oal_level_device_state(oal_level* L, void** f, void** rho, void** vel);
/* Bytes of device memory this level holds. */
int64_t oal_level_device_bytes(const oal_level* L);
/* D3Q39 entropic levels (operator OAL_OP_ENTROPIC_D3Q39, storage OAL_STORE_F32, a library-built
 * geometry with no sponge and no wall distance within 16 cells; domain faces and solid cells are
 * taken as the reference's default boundary options and full-way bounce-back): the
 * 13-multiplier warm-start cache of the equilibrium solve (timestep.jl:1447-1450), host float in
 * the reference layout lambda(8,8,8,n_blocks,13), NaN = no warm start. get_host receives the
 * cache, set_host (after the get) replaces it; either may be NULL. Init and set_state reset it to
 * NaN, as the reference allocates it. Synchronises. */
oal_status oal_level_entropic_lambda(oal_level* L, float* get_host, const float* set_host);
/* Population layout of the level's device state (what oal_level_device_state points at):
 * out = {dense, PX, PY, PZ, block_stride, dir_stride}. dense = 1: box levels in FP32/FP16/BF16
 * keep f[k][Z][Y][X] on a padded PX x PY x PZ grid (interior cell (i,j,l) at X = i+8, Y = j+1,
 * Z = l+1); dense = 0: block-major f[b][k][cell], element b*block_stride + k*dir_stride + cell. */
oal_status oal_level_layout(const oal_level* L, int64_t out[6]);

/* ---- block AMR: D3Q27 levels with 2:1 refinement in space and time --------------------------
 * Replaces recursive_step! / recursive_step_temporal! / execute_timestep_batch!
 * (src/solver/solver_control.jl:55-828), the refined levels' parent interpolation
 * interpolate_with_rescaling (src/collision/physics_interpolation.jl:705-1198, called from
 * kernel_cumulant.jl:286-316,346-388) and restrict_fine_to_parent! (src/collision/amr_coupling.jl:
 * 7562-8035, kernel :1900-3242), at the reference's default settings: temporal interpolation on (the
 * parent's state before and after its step, child substeps at weights 0 and 1/2), cubic Lagrange
 * macros and f_neq with the extrapolating trilinear fallback, the post-collision f_neq factor, the
 * children-average restriction with two moment-correction passes. Level l (0-based) has a block grid
 * of 2^l x the coarse one and a geometry whose nx/ny/nz are 8 x that grid (its cells at its own
 * resolution; domain faces apply at every level); every block of level l > 0 lies inside a block of
 * level l - 1. A coarse step steps level 0 once, then (recursively) each finer level twice, then
 * restricts it onto its parent. */
typedef struct oal_amr oal_amr;
typedef struct oal_amr_level_desc {
  const oal_geometry* geometry;  /* the level's blocks (coordinates in its block grid, 1-based) */
  int32_t dim[3];                /* block-grid extent of the level */
  int32_t reserved;
} oal_amr_level_desc;
oal_status oal_amr_create(int32_t nlevels, const oal_amr_level_desc* levels, int32_t storage, oal_amr** out);
void oal_amr_destroy(oal_amr* A);
/* The state of level `level` (0 = coarsest), owned by the hierarchy: initialise, read or write it with
 * the oal_level_* calls (init_equilibrium, get_state, set_state, mass_momentum, get_forces). */
oal_status oal_amr_level(oal_amr* A, int32_t level, oal_level** out);
/* n coarse steps as one CUDA graph; params[l] are level l's step parameters (tau per level). */
oal_status oal_amr_advance(oal_amr* A, const oal_step_params* params, int32_t n_coarse_steps, void* stream);

/* ---- batches: many cases stepped by one launch per kernel ------------------------------------ */
/* A batch owns a block pool (populations in `storage`, macros, masks) and steps every member case
 * with one launch per kernel per step; n steps are one CUDA graph. Members are added and removed
 * between advances without moving other members' state; each result is independent of the batch
 * composition (per-case parameters, per-case fixed-order FP64 reductions). The reference runs
 * cases one after another (src/main.jl:2184-2238); this is the batched form of
 * execute_timestep_batch! (src/solver/solver_control.jl:796-828). */
typedef struct oal_batch oal_batch;
oal_status oal_batch_create(int32_t device, int32_t storage, int32_t max_real_blocks, int32_t max_ghost_blocks,
                            int32_t max_mask_blocks, int32_t max_members, oal_batch** out);
void oal_batch_destroy(oal_batch* B);
/* Admit a case (block-layout geometry on the batch's device, its step parameters, equilibrium start
 * from host rho(8,8,8,nb) / vel(8,8,8,nb,3) in double). OAL_E_ADMISSION when the pool has no room. */
oal_status oal_batch_add(oal_batch* B, const oal_geometry* g, const oal_step_params* p, const double* rho_host,
                         const double* vel_host, int32_t* member_out);
oal_status oal_batch_remove(oal_batch* B, int32_t member);
oal_status oal_batch_set_params(oal_batch* B, int32_t member, const oal_step_params* p);
/* a member's linear Bouzidi boundary cells (as oal_level_set_bouzidi, block indices of the
 * member's geometry); the member's steps with solid_bc OAL_SOLID_BOUZIDI apply them */
oal_status oal_batch_set_bouzidi(oal_batch* B, int32_t member, int32_t n_cells, const int32_t* cell_block,
                                 const int32_t* cell_x, const int32_t* cell_y, const int32_t* cell_z,
                                 const uint16_t* q_half, float q_min_threshold, int32_t ff_fallback,
                                 float limiter_rel_cap, float limiter_abs_cap);
oal_status oal_batch_advance(oal_batch* B, int32_t n_steps, void* stream);
/* Launch tuning of the pool's kernels (OAL_TUNE_* keys as for levels) and the autotuner over the
 * current members: each candidate advances n_steps from the pool's current state, which is
 * restored afterwards. */
oal_status oal_batch_set_tuning(oal_batch* B, int32_t key, int64_t value);
oal_status oal_batch_get_tuning(const oal_batch* B, int32_t key, int64_t* value);
oal_status oal_batch_autotune(oal_batch* B, int32_t n_steps, int64_t* prefetch, int32_t* persistent,
                              double* ms_per_step);
/* Member state in the reference layout (double); synchronises. Any pointer may be NULL. */
oal_status oal_batch_get_state(oal_batch* B, int32_t member, double* f, double* rho, double* vel);
/* Momentum-exchange force of the member's last collecting step (FP64, lattice units); synchronises. */
oal_status oal_batch_get_forces(oal_batch* B, int32_t member, double out[3]);
oal_status oal_batch_mass_momentum(oal_batch* B, int32_t member, double out[4]);
/* Pool usage: out = {members, real blocks used, ghost blocks used, mask blocks used,
 * real capacity, ghost capacity, mask capacity, device bytes}. */
oal_status oal_batch_info(const oal_batch* B, int64_t out[8]);
/* Blocks one member of this geometry occupies: out = {real, ghost, mask}. */
oal_status oal_geometry_blocks(const oal_geometry* g, int64_t out[3]);

/* ---- no-allocation entry point -------------------------------------------------------------- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc when they need the
 * totals (a stream-ordered pool that forbids stray allocations, a host runtime such as a Julia
 * task on CUDA.jl's allocator that must not grow device memory between steps): FP64 {mass, px,
 * py, pz} of the fluid cells of caller-owned populations, with the per-block partial sums kept in
 * a fixed file-scope device array of OAL_NOALLOC_MAX_BLOCKS blocks (2 MiB, held by every GPU that
 * loads the library until the process exits). f: device populations (storage type, element
 * strides as in oal_level_fields); obstacle: device uint8[512*n_blocks] or NULL; out: device
 * double[4]. n_blocks above the maximum returns OAL_E_TOO_LARGE. The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) and should come before any stream capture.
 * All calls share the array: calls that overlap on the GPU race and must be serialised. The
 * looked-up address is kept per device number for the life of the process: after a
 * cudaDeviceReset (or any new primary context) on that device the kept address is stale, so a
 * process that resets a device must not call this entry point on it again. */
#define OAL_NOALLOC_MAX_BLOCKS 65536
oal_status oal_mass_momentum_noalloc(const void* f, int32_t storage, int64_t f_block_stride, int64_t f_dir_stride,
                                     const uint8_t* obstacle, int32_t n_blocks, double* out, void* stream);

/* ---- D3Q19 octree level (OpenAeroLab src/octree_q19) -----------------------------------------
 *
 *   reference                                              replaced by
 *   -----------------------------------------------------  ------------------------------------
 *   Numerics (nu per level, sgs, c_wale, c_smagorinsky,    oal_q19_params / oal_q19_default_params
 *     hrr_sigma, body_force) config.jl:306-335,
 *     state.jl:235-249
 *   generate(Tri[], MeshSpec(periodic=(true,true,true),    oal_q19_periodic_box
 *     levels=1)) generator.jl:270-350 (level 1 of a
 *     periodic box: octs in Morton order, onbr)
 *   State(mesh, cfg, T) level buffers f/g, u/v, rho/rhob   oal_q19_level_create / _destroy
 *     state.jl:40-60,230-255
 *   initialise!(st, init) / initialise_uniform!            oal_q19_level_initialise
 *     state.jl:267-330 (host evaluates init; rebuild on the device)
 *   advance!(st) = step_level! + swap_buffers!             oal_q19_level_advance
 *     run.jl:6-11, stream.jl:280-380
 *   total_mass / total_momentum (Float64)                  oal_q19_level_totals
 *     state.jl:333-356
 *   generate(tri, MeshSpec(levels=1)) generator.jl:106-837 oal_q19_mesh_generate / _counts / _level_desc
 *   State(mesh, cfg, T) on a mesh with a body              oal_q19_level_create_desc
 *   st.forces after advance!(st; collect=true)             oal_q19_level_forces
 *     stream.jl:248-256, run.jl reduce_forces!
 *   collide_rr(f, omega, sigma, pi_fd, F) per cell         oal_q19_collide_cells (test hook)
 *     collision.jl:58-75, kernel.jl:92-134
 *
 * Layouts (Julia column-major, the reference's own): f(8,19,nocts) shifted populations f - w_i,
 * u(8,3,nocts), rho(8,nocts), du(8,9,nocts) with du[k, 3a+b, o] = d u_b / d x_a over one cell,
 * onbr(27,nocts) 1-based (0 = none), origin(3,nocts) 0-based level cells. `precision` is
 * OAL_STORE_F32 or OAL_STORE_F64 (the solver's Float32 / Float64); host arrays have that type.
 * Octs of a periodic level made by oal_q19_level_create must have all 26 neighbours; levels with
 * domain faces and bodies come through oal_q19_level_create_desc. Refinement (ghost / covered
 * slots, several levels) is refused with OAL_E_UNSUPPORTED. */
enum { OAL_Q19_SGS_NONE = 0, OAL_Q19_SGS_WALE = 1, OAL_Q19_SGS_SMAGORINSKY = 2, OAL_Q19_SGS_VREMAN = 3 };

typedef struct oal_q19_params {
  uint32_t abi_version;   /* OAL_ABI_VERSION */
  int32_t sgs;            /* OAL_Q19_SGS_* */
  double nu;              /* molecular viscosity, lattice units of the level */
  double c_wale;          /* WALE constant (0.5) */
  double c_smagorinsky;   /* Smagorinsky constant (0.1); Vreman uses 2.5 c^2 */
  double hrr_sigma;       /* 1 = RR; < 1 blends the finite-difference stress (HRR) */
  double body_force[3];   /* Guo body force, lattice units of the level */
  double u_inlet[3];      /* inlet / freestream velocity of the open faces, lattice units (stream.jl:291) */
  double force_scale;     /* momentum-exchange scale of the level, 8^(1-l) (1 on a single level) */
} oal_q19_params;

/* Slot kinds (octree.jl:5-11) and domain-face conditions (MeshSpec.faces, generator.jl:29). */
enum { OAL_Q19_K_NONE = 0, OAL_Q19_K_FLUID = 1, OAL_Q19_K_SOLID = 2, OAL_Q19_K_COVERED = 3, OAL_Q19_K_GHOST = 4,
       OAL_Q19_K_BOUNDARY = 5 };
enum { OAL_Q19_FACE_PERIODIC = 0, OAL_Q19_FACE_INLET = 1, OAL_Q19_FACE_OUTLET = 2, OAL_Q19_FACE_SLIP = 3,
       OAL_Q19_FACE_SYMMETRY = 4, OAL_Q19_FACE_NOSLIP = 5, OAL_Q19_FACE_GROUND = 6, OAL_Q19_FACE_FREESTREAM = 7 };

/* One level of an octree mesh, the reference's OctLevel arrays (octree.jl:50-71), all host memory,
 * 1-based indices as in the reference. Nullable: real (all real), kind (all fluid), face, special
 * and cutidx (none), the cut arrays when ncut = 0, the transfer lists when their count is 0. */
typedef struct oal_q19_level_desc {
  int32_t nocts;
  const int32_t* origin;       /* (3, nocts) level cells */
  const uint8_t* real;         /* (nocts) stepped octs */
  const int32_t* onbr;         /* (27, nocts) */
  const uint8_t* kind;         /* (8, nocts) OAL_Q19_K_* */
  const uint8_t* face;         /* (8, nocts) faces a boundary slot lies beyond, bit f = face f (-x +x -y +y -z +z) */
  const uint32_t* special;     /* (8, nocts) bit j-1: direction j arrives by a face condition or a cut link */
  const int32_t* cutidx;       /* (8, nocts) cut cell of a fluid slot, 0 none */
  int32_t ncut;                /* cut cells */
  const int32_t* cut_slot;     /* (ncut) slot id k + 8 (o - 1) */
  const int32_t* cut_off;      /* (ncut + 1) CSR into the links */
  int32_t nlinks;
  const uint8_t* cut_dir;      /* (nlinks) direction 2..19 toward the wall */
  const float* cut_q;          /* (nlinks) Bouzidi q in (0, 1] */
  const int32_t* cut_tri;      /* (nlinks) triangle, 0 none */
  const uint8_t* cut_partner;  /* (nlinks) the Bouzidi partner x - c_i is a plain fluid slot */
  int32_t ntri;                /* triangles (force bins) */
  int32_t faces[6];            /* OAL_Q19_FACE_* of -x +x -y +y -z +z */
  /* transfers between levels (generator.jl:600-790): the ghost slots of this level filled from the
   * coarser level (64 donor slots of level-1 with weights per ghost), and the covered slots of this
   * level restricted from the finer one (64 source slots of level+1, cubic or inner-8 average) */
  int32_t nghost;
  const int32_t* ghost_slot;   /* (nghost) */
  const int32_t* ghost_donor;  /* (64, nghost) slot ids of the coarser level, 0 unused */
  const float* ghost_w;        /* (64, nghost) */
  int32_t nrestrict;
  const int32_t* restrict_slot;   /* (nrestrict) */
  const int32_t* restrict_src;    /* (64, nrestrict) slot ids of the finer level, 0 unused */
  const uint8_t* restrict_cubic;  /* (nrestrict) */
} oal_q19_level_desc;

/* A refinement region of the mesh spec (generator.jl:10-16). */
typedef struct oal_q19_region {
  int32_t kind;                /* 0 box (lo..hi), 1 sphere (centre, radius), 2 cylinder (axis lo -> hi, radius) */
  int32_t level;               /* refined up to this level */
  double lo[3], hi[3], centre[3], radius;
} oal_q19_region;

/* a box of its own surface level (SurfaceLevel, generator.jl:18-21): cells whose centre lies in
 * [lo, hi] take max(surface_level, level) as their surface level */
typedef struct oal_q19_surface_level {
  int32_t level;
  double lo[3], hi[3];
} oal_q19_surface_level;

/* MeshSpec (generator.jl:21-36). */
typedef struct oal_q19_mesh_spec {
  double domain[3];            /* metres; periodic axes an even number of coarse cells */
  double dx;                   /* finest cell size, metres */
  int32_t periodic[3];
  int32_t faces[6];            /* OAL_Q19_FACE_*, PERIODIC exactly on periodic axes */
  int32_t levels;              /* L >= 1 */
  int32_t surface_level;       /* level of the surface band (0 = L) */
  int32_t band_fine;           /* band of the surface level, its cells (8) */
  int32_t band;                /* band of each coarser level, its cells (6) */
  int32_t wake_level_offset;   /* wake level = surface_level - offset (1) */
  double wake_length;          /* body x extents; 0 disables */
  double wake_margin;          /* body extents (0.1) */
  int32_t nregions;
  const oal_q19_region* regions;
  /* seal_cavities (generator.jl:37, 383-414, off by default): fluid slots inside the body's
   * bounding box (one coarsest cell of margin) that axis-ray parity puts inside the surface stay
   * out of the flood fill, so the interior of a leaky model stays solid */
  int32_t seal_cavities;
  int32_t nsurface_levels;     /* per-box surface levels (generator.jl:35, 185) */
  const oal_q19_surface_level* surface_levels;
  int32_t reserved[2];
} oal_q19_mesh_spec;
typedef struct oal_q19_mesh oal_q19_mesh;

typedef struct oal_q19_level oal_q19_level;

oal_status oal_q19_default_params(oal_q19_params* out);
oal_status oal_q19_periodic_box(int32_t n0, int32_t n1, int32_t n2, int32_t* origin, int32_t* onbr);
oal_status oal_q19_default_mesh_spec(oal_q19_mesh_spec* out);
/* tri: (ntri, 3 vertices, 3 coordinates) metres; ntri = 0 meshes an empty box */
oal_status oal_q19_mesh_generate(const double* tri, int32_t ntri, const oal_q19_mesh_spec* spec, oal_q19_mesh** out);
oal_status oal_q19_mesh_destroy(oal_q19_mesh* mesh);
int32_t oal_q19_mesh_levels(const oal_q19_mesh* mesh);
/* counts of level `level` (1..L): out[16] = {nocts, n0, n1, n2, fluid, solid, boundary, cut cells,
 * cut links, leak cells, links without a Bouzidi partner, unreached triangles, special slots,
 * real octs, listed ghosts, restricted slots}; level 0: the same summed over the levels (n0..n2
 * of the finest level, the leak / unreached / triangle counts of the mesh) */
oal_status oal_q19_mesh_counts(const oal_q19_mesh* mesh, int32_t level, int64_t* out);
/* the cavity-sealing report of the mesh (generator.jl:411-412): out[2] = {sealed_cells,
 * cavity_unbracketed_parity_cells} (both 0 without seal_cavities) */
oal_status oal_q19_mesh_seal_counts(const oal_q19_mesh* mesh, int64_t* out);
/* level `level` (1..L) as a descriptor (pointers valid while the mesh lives) */
oal_status oal_q19_mesh_level_desc(const oal_q19_mesh* mesh, int32_t level, oal_q19_level_desc* out);

oal_status oal_q19_level_create(int32_t device, int32_t precision, int32_t nocts, const int32_t* onbr,
                                oal_q19_level** out);
oal_status oal_q19_level_create_desc(int32_t device, int32_t precision, const oal_q19_level_desc* desc,
                                     oal_q19_level** out);
oal_status oal_q19_level_destroy(oal_q19_level* level);
/* host rho, u and (nullable) du: with du the Chapman-Enskog non-equilibrium is rebuilt, else the equilibrium */
oal_status oal_q19_level_initialise(oal_q19_level* level, const oal_q19_params* p, const void* rho, const void* u,
                                    const void* du);
/* n steps; with collect_forces the last step accumulates the momentum exchange of the cut links
 * (stream.jl:248-256), read by oal_q19_level_forces */
oal_status oal_q19_level_advance(oal_q19_level* level, const oal_q19_params* p, int32_t n_steps,
                                 int32_t collect_forces, void* stream);
/* FP64 force on the walls of the last collecting step: total[3], and per triangle (ntri, 3) if not null
 * (links without a triangle count to triangle 1, as run.jl's accumulator does) */
oal_status oal_q19_level_forces(oal_q19_level* level, double* total, double* per_triangle);
oal_status oal_q19_level_get_state(oal_q19_level* level, void* f, void* u, void* rho);       /* host, nullable */
oal_status oal_q19_level_set_state(oal_q19_level* level, const void* f, const void* u, const void* rho);
/* either population/macro buffer: which 0 = the current one (the reference's S.f, S.u, S.rho),
 * 1 = the other (S.g, S.v, S.rhob: the previous step's, which the time blend of a refined mesh's
 * ghost fill reads); host, nullable on get */
oal_status oal_q19_level_get_buffer(oal_q19_level* level, int32_t which, void* f, void* u, void* rho);
oal_status oal_q19_level_set_buffer(oal_q19_level* level, int32_t which, const void* f, const void* u, const void* rho);
oal_status oal_q19_level_device_state(oal_q19_level* level, void** f, void** u, void** rho, int64_t* steps);
/* out[5] = {mass, px, py, pz, kinetic energy sum 0.5 rho |u|^2}, FP64, fixed reduction order */
oal_status oal_q19_level_totals(oal_q19_level* level, double* out, void* stream);
/* device arrays: f(n,19) omega(n) pfd(n,6) F(n,3) -> out(n,19) rho(n) u(n,3) */
/* ---- several levels: the recursive step (run.jl:6-11, coupling.jl step_recursive!) ----------
 * One coarse step = one step of level 1 and, recursively, two of each finer level, with the
 * restriction into the covered slots and the ghost fill at the half and full time (coupling.jl).
 * `params` holds one oal_q19_params per level (nu, body force and force scale of that level's
 * lattice units). Level l's arrays are read through oal_q19_octree_level. */
typedef struct oal_q19_octree oal_q19_octree;
oal_status oal_q19_octree_create(int32_t device, int32_t precision, int32_t nlevels, const oal_q19_level_desc* levels,
                                 oal_q19_octree** out);
oal_status oal_q19_octree_destroy(oal_q19_octree* tree);
oal_status oal_q19_octree_level(oal_q19_octree* tree, int32_t level, oal_q19_level** out);
/* per level host arrays rho[l], u[l], du[l] (du[l] nullable) for the fluid, ghost and covered slots;
 * then the coupling of the initial state (couple_initial!) */
oal_status oal_q19_octree_initialise(oal_q19_octree* tree, const oal_q19_params* params, const void* const* rho,
                                     const void* const* u, const void* const* du);
oal_status oal_q19_octree_advance(oal_q19_octree* tree, const oal_q19_params* params, int32_t n_coarse_steps,
                                  int32_t collect_forces, void* stream);
/* force of the last collecting coarse step over all levels and sub-steps, coarse-lattice units */
oal_status oal_q19_octree_forces(oal_q19_octree* tree, double* total, double* per_triangle);
/* FP64 {mass, px, py, pz, kinetic energy} over the fluid leaves, each level weighted by 8^(L-l) */
oal_status oal_q19_octree_totals(oal_q19_octree* tree, double* out);

oal_status oal_q19_collide_cells(int32_t precision, int64_t n, const void* f, const void* omega, double sigma,
                                 const void* pfd, const void* F, void* out, void* rho, void* u, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OAL_H */
