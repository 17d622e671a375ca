// common.cuh — shared device definitions of liboal: the D3Q27 velocity set as compile-time
// constants, the population storage codecs and the argument blocks of the step kernels.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace oal {

constexpr int kQ27 = 27;
constexpr int kBS = 8;           // block edge (src/geometry/blocks.jl:14)
constexpr int kCells = 512;      // cells per block

// D3Q27 ordering of the reference (src/collision/lattice.jl:16, z outer, x inner):
// k = (cx+1) + 3(cy+1) + 9(cz+1), 0-based here. The chimera passes rely on this order.
__host__ __device__ constexpr int q27_cx(int k) { return k % 3 - 1; }
__host__ __device__ constexpr int q27_cy(int k) { return (k / 3) % 3 - 1; }
__host__ __device__ constexpr int q27_cz(int k) { return k / 9 - 1; }
__host__ __device__ constexpr int q27_opp(int k) { return 26 - k; }
__host__ __device__ constexpr int q27_mir_y(int k) { return (k % 3) + 3 * (2 - (k / 3) % 3) + 9 * (k / 9); }
__host__ __device__ constexpr int q27_mir_z(int k) { return (k % 9) + 9 * (2 - k / 9); }
__host__ __device__ constexpr int q27_d2(int k) {
  return q27_cx(k) * q27_cx(k) + q27_cy(k) * q27_cy(k) + q27_cz(k) * q27_cz(k);
}
// weights 8/27, 2/27, 1/54, 1/216 by |c|^2 (lattice.jl:22-31)
__host__ __device__ constexpr double q27_w(int k) {
  return q27_d2(k) == 0 ? 8.0 / 27.0 : q27_d2(k) == 1 ? 2.0 / 27.0 : q27_d2(k) == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
}
// direction index of a neighbour-block offset (ox,oy,oz) in {-1,0,1}^3 (domain_topology.jl:940)
__host__ __device__ constexpr int nbr_dir(int ox, int oy, int oz) { return (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1); }

// ---- population storage codecs --------------------------------------------------------------
// F32/F64: the population itself. F16/BF16 "deviation": d = f/w_k - 1, so that every direction
// stores an O(Ma) number and the half-precision relative rounding applies to the deviation only.
template <class S> struct Codec;
template <> struct Codec<float> {
  template <class R> __device__ static __forceinline__ R dec(float v, R, R) { return R(v); }
  template <class R> __device__ static __forceinline__ float enc(R f, R, R) { return float(f); }
};
template <> struct Codec<double> {
  template <class R> __device__ static __forceinline__ R dec(double v, R, R) { return R(v); }
  template <class R> __device__ static __forceinline__ double enc(R f, R, R) { return double(f); }
};
template <> struct Codec<__half> {
  __device__ static __forceinline__ float dec(__half v, float w, float) { return fmaf(w, __half2float(v), w); }
  __device__ static __forceinline__ __half enc(float f, float, float inv_w) { return __float2half_rn(fmaf(f, inv_w, -1.0f)); }
};
template <> struct Codec<__nv_bfloat16> {
  __device__ static __forceinline__ float dec(__nv_bfloat16 v, float w, float) { return fmaf(w, __bfloat162float(v), w); }
  __device__ static __forceinline__ __nv_bfloat16 enc(float f, float, float inv_w) { return __float2bfloat16_rn(fmaf(f, inv_w, -1.0f)); }
};

// ---- per-case scalar parameters (resolved from oal_step_params on the host) -----------------
enum CaseFlags : uint32_t {
  CF_ADAPTIVE_OMEGA4 = 1u << 0,
  CF_LIMITER_FACTORED = 1u << 1,
  CF_LIMITER_POSITIVITY = 1u << 2,
  CF_COMPRESSIBLE = 1u << 3,
  CF_YMIN_WALL = 1u << 4,
  CF_ZWALL_SLIP = 1u << 5,
  CF_ZWALL_NOSLIP = 1u << 6,
  CF_WALL_MODEL = 1u << 7,
  CF_SPONGE_BLEND = 1u << 8,
  CF_TRANSVERSE_FS = 1u << 9,
  CF_HALFWAY = 1u << 10,
  CF_COLLECT = 1u << 11,
  CF_STORE_POST = 1u << 12,
  CF_GRADIENTS = 1u << 13,  // c_wale != 0: the WALE velocity-gradient stencil is needed
  CF_INLET_NOISE = 1u << 14,
  CF_PERIODIC_X = 1u << 15,  // periodic axes of a dense (box) level
  CF_PERIODIC_Y = 1u << 16,
  CF_PERIODIC_Z = 1u << 17,
  CF_GRAD_WALL = 1u << 18,   // Grad-reconstruction wall on fluid cells with links into solids
  CF_BOUZIDI = 1u << 19,     // linear Bouzidi correction after the step (the step itself is full-way)
  CF_GENERAL_RATES = 1u << 20, // omega_bulk, omega3 or omega4 differs from 1 (the configuration default)
  CF_SGS_PI = 1u << 21,        // variable nu_sgs from the stored post-collision Pi_neq
  CF_SGS_DYNAMIC = 1u << 22    // variable nu_sgs from the Germano-Lilly dynamic coefficient
};

struct CaseParams {
  float tau, c_wale, nu_sgs_bg, amr_sgs_scale;
  float omega_bulk, omega3, omega4, lambda_param;
  float u_inlet, inlet_turbulence, wall_model_max_distance, transverse_blend;
  int32_t time_step_seed;
  uint32_t flags;
  int32_t nx, ny, nz;
  float grad_pineq_scale;  // CF_GRAD_WALL
  float c_pi, nu_sgs_floor;  // CF_SGS_PI / CF_SGS_DYNAMIC
};
static_assert(sizeof(CaseParams) == 80, "CaseParams layout");

// per-block geometry flags
enum BlockFlags : uint32_t {
  BF_INTERIOR = 1u << 0,    // all 26 neighbour blocks exist: no domain-face pulls
  BF_NEAR_SOLID = 1u << 1,  // per-cell solid masks apply (own or a pull source is solid)
};

// Kernel argument block of one launch. Element strides address either the reference layout
// (block stride 512, direction stride 512*n_blocks) or the block-major layout of library-owned
// state (block stride 512*Q, direction stride 512).
// The parent level seen from a refined level (block AMR, perform_timestep_v2!'s parent_* arguments):
// pulls from outside the level's blocks but inside the domain are interpolated from it. ptr == null
// on level 1.
struct ParentView {
  const void* f_new;    // storage type, block-major (block stride 27*512, direction stride 512)
  const void* f_old;    // the same before the parent's step, or null
  const void* rho_new;  // compute type, [nb*512]
  const void* rho_old;
  const void* vel_new;  // compute type, component stride nb*512
  const void* vel_old;
  const int32_t* ptr;   // [dim_x*dim_y*dim_z], x fastest: 1-based parent block, 0 = none
  int32_t dim_x, dim_y, dim_z, nb;
  double tau_parent, tau_fine, tw;
  int32_t use_temporal, level_visc_physical;
  // parent nodes evaluated once per substep (k_parent_nodes): node_map[parent cell] = record index
  // or -1; record = 32 values of the compute type: blended rho, ux, uy, uz, then f_neq of the 27
  // directions. Null: evaluate nodes on the fly.
  const int32_t* node_map;
  const void* node_vals;
  // interpolation positions (the level's ghost cells whose pulls interpolate): slot_pos[(ghost
  // block - real blocks) * 512 + cell] = position or -1; pos_nodes[position * 64 + 16(a+1) +
  // 4(b+1) + (c+1)] = record of parent node (px0+a, py0+b, pz0+c) or -1 (absent); pos_macro =
  // the interpolated rho, ux, uy, uz of each position (k_parent_positions, once per substep)
  const int32_t* slot_pos;
  const int32_t* pos_nodes;
  const void* pos_macro;
  int32_t n_pos, n_real;
};

// Restriction of a child level onto its parent (block AMR)
struct RestrictArgs {
  void* pf;                 // parent's current populations (storage type), block-major
  void* prho;               // parent's density (compute type), [pnb*512]
  void* pvel;               // parent's current velocity, component stride pnb*512
  const int4* pbinfo;       // parent block coordinates (1-based)
  const int32_t* covered;   // parent blocks that have children
  int32_t n_covered, pnb;
  const void* cf;           // child's current populations (storage type), block-major
  const int32_t* cptr;      // child block pointer [cdx*cdy*cdz], x fastest, 1-based, 0 = none
  int32_t cdx, cdy, cdz;
  const uint32_t* cbflags;  // child solid masks (BF_NEAR_SOLID blocks, bit 13 = own cell solid)
  const int32_t* cmslot;
  const uint32_t* ccmask;
  double ratio;             // tau ratio of the f_neq rescale (with the post-collision factor)
  int32_t comp;
};

struct StepArgs {
  const void* f_in;
  void* f_out;
  void* f_post;
  void* rho_out;
  void* vel_out;
  const void* vel_in;
  int64_t f_bstride, f_kstride;
  int64_t v_bstride, v_cstride;   // velocity/density: block stride, component stride
  const int32_t* nbr;             // [nb*27], 0-based block index, -1 = none
  const int4* binfo;              // [nb] (bx, by, bz, case) 1-based coords
  const uint32_t* bflags;         // [nb]
  const int32_t* mslot;           // [nb] mask slot or -1
  const uint32_t* cmask;          // [slots*512] bit k: source of direction k is solid (13: own)
  const float* sponge;            // [nb*512] or null
  const float* wall_dist;         // [nb*512] or null
  const CaseParams* cases;        // [n_cases] or null (use p0)
  double* force_part;             // [n_ctas*3] momentum-exchange partials or null
  int32_t n_blocks;
  int32_t block_base;             // first block of this launch (per-case launches)
  int32_t n_total_blocks;         // real + ghost blocks of the population buffers
  // dense (box) population layout: f[k][Z][Y][X] over a padded grid PX x PY x PZ with the
  // interior cell (i,j,l) at X = i + 8, Y = j + 1, Z = l + 1; f_kstride = PX*PY*PZ
  int32_t dense;
  int32_t PX, PY, PZ;
  uint32_t* err;                  // device error word (bounded waits that gave up), or null
  uint32_t flags_any;             // OR of the flags of every case of the launch (kernel selection)
  int32_t round_nearest;          // 16-bit codecs: round stored deviations to nearest (else stochastically)
  int32_t prefetch_ctas;          // x-pair kernel: CTA j also prefetches CTA j + prefetch_ctas's
                                  // populations and velocities into L2 (0 = off; launch tuning)
  int32_t persistent;             // x-pair kernel: resident CTAs walk the units (launch tuning)
  int32_t pairs_units;            // set by the launcher: units of a persistent launch (0 = one per CTA)
  const int32_t* fast_rec;        // x-pair kernel: per work entry 32 ints (27-entry neighbour row,
                                  // block coordinates + case, block index), in work-list order
  void* pi_neq;                   // CF_SGS_PI: post-collision Pi_neq (compute type, [6][nb*512]),
                                  // read at the cell, then rewritten with this step's
  double* force_out;              // general kernel of a single level: the last CTA sums the
  uint32_t* force_ticket;         // momentum-exchange partials into force_out (ticket reset to 0)
  CaseParams p0;
  ParentView par;                 // refined levels only (par.ptr == null otherwise)
};

// Bulk prefetch of [p, p + bytes) from global memory into L2 (no register result, no wait): the
// address and the size are multiples of 16 bytes.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(bytes) : "memory");
}

// Element index of cell (X, Y, Z) of the dense padded population grid (direction 0).
__host__ __device__ __forceinline__ int64_t dense_idx(const StepArgs& a, int X, int Y, int Z) {
  return ((int64_t)Z * a.PY + Y) * a.PX + X;
}

// Element index of (block b, cell, direction k) in either population layout of a level.
struct PopIndex {
  const int4* binfo;
  int dense;
  int PX, PY;
  int64_t bst, kst;
  __device__ __forceinline__ int64_t operator()(int64_t b, int cell, int k) const {
    if (dense) {
      const int4 bi = binfo[b];
      const int X = (bi.x - 1) * kBS + (cell & 7) + 8, Y = (bi.y - 1) * kBS + ((cell >> 3) & 7) + 1,
                Z = (bi.z - 1) * kBS + (cell >> 6) + 1;
      return ((int64_t)Z * PY + Y) * PX + X + k * kst;
    }
    return b * bst + k * kst + cell;
  }
};

}  // namespace oal
