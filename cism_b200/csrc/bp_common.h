// bp_common.h -- types shared by the host plan builder and the device kernels.
//
// Device data model.  A solve (or a batch of independent solves) is
// compiled into a set of *columns*: the locally owned, active vertices of
// each instance (the rows the reference's matvec computes,
// glissade_velo_higher_pcg.F90:2605-2612).  The halo of the reference's
// local grid disappears: a periodic image map turns halo vertices into the
// owned vertices they copy (parallel_slap.F90:2807-2925), so every stencil
// neighbour is an owned column or absent.  Levels k = 0 (the upper surface)
// to nz-1 (the bed), as in the reference.  Node layout: each instance's
// columns are cut into blocks of W consecutive columns (W a power of two,
// W * nz <= kTile), and a block's nodes are stored level-major, node
// (col, k) = col_node[col] + k * W, so that consecutive columns at one
// level are consecutive in memory: a warp reading 32 columns of a level
// reads contiguous vectors and coefficients, and a column's levels are W
// apart.  Blocks never span two instances; the slots of an instance's last
// block past its columns are holes that no kernel touches.  Elements are
// the reference's active cells (i,j in [nhalo+1, n-nhalo+1]) times nz-1
// layers; their geometry is taken from the halo'd vertex arrays so periodic
// surface offsets are preserved.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define BP_HD __host__ __device__ __forceinline__
#include <cuda_runtime.h>
#else
#define BP_HD inline
#include <vector_types.h>  // double2 / float2 (plain structs under a host compiler)
#endif

namespace bp {

constexpr int kNzMax = 64;     // largest supported number of levels
constexpr int kTile = 256;     // nodes per tile; one CTA of kTile threads per tile
constexpr double kVol0 = 1.0e9;  // volume scale, glissade_velo_higher.F90:1111

// Velocity-dependent sliding law of an instance (calcbeta,
// glissade_basal_traction.F90:67-598), law = which_ho_babc; 0 = none
// (beta fixed over the Picard loop).  The exponents and the products of
// constants the law evaluates before the speed enters are formed on the
// host; per-column products live in DevView::col_slide.
struct SlideParams {
  int law;
  double umax;   // beta_powerlaw_umax (<= 0: no cap)
  double bmin;   // beta_grounded_min
  double c;      // powerlaw_c (laws 9, 12)
  double e1;     // law 3: 1 - q; 10: 1/gn - 1; 11, 12: 1/m; 13: 1/p - 1
  double e2;     // law 9, 11: 1/m - 1; 10: -1/gn
  double k;      // law 3: u0^q; 11: powerlaw_c^m
};

// Per-instance constants (read-only on the device).
struct InstParams {
  double dx, dy;
  double efvs_constant;
  double pcg_tol;
  double inner_tol;
  double sigma[kNzMax];
  int which_efvs, which_babc, which_assemble_beta, which_resid;
  int precond, variant, precision;
  int pcg_maxiters, ncheck, maxiter_nonlinear;
  int col_begin, col_end;
  int node_begin, node_end;
  int tile_begin, tile_end;
  int cell_begin, cell_end;
  int elem_begin, elem_end;
  SlideParams slide;
  double rhoi, grav;            // L1L2: tau_perp = rhoi grav depth |grad s|
};

// Per-instance solver state (device-resident, written by finalizers).
struct InstState {
  double bb, L2_rhs;            // (b,b) and its root
  double rz, rz_old;            // eta1 / eta0 (standard) ; rho / rho_old (Chron-Gear)
  double alpha, beta, sigma;    // CG scalars
  double err;                   // |b-Ax|/|b| at the last check
  double L2_norm, L2_rel;       // residual before the linear solve
  double resid_velo;            // Picard criterion value
  double r_true;                // mixed: |b - A x| at the last refinement
  int pcg_iter, pcg_active, pcg_converged;
  int picard_iter, picard_active, picard_converged;
  int status;                   // bp_status
  int nonzero;                  // any nonzero matrix entry (count_nonzeros_3d)
  int zero_x;                   // velocity must be zeroed (all-zero matrix)
  int pcg_iters_total, pcg_iters_last;
  int refine_active, refine_steps, refine_steps_total;
  int inner_iter;
  int krylov_fp64;              // mixed: Krylov matvecs switched to the FP64 matrix
  int need_true;                // mixed: the next check computes the FP64 residual
  int restart;                  // mixed, Chronopoulos-Gear: next pass restarts (beta = 0)
  int last_true_iter;           // mixed: pcg_iter of the last refinement
  int frozen;                   // 2-D solve on a no-slip bed: 2-D velocity zero, no linear solve
};

// Global counters polled by the host.
struct Counters {
  int pcg_active;
  int picard_active;
  int refine_active;
  int pad;
};

// Device view of a compiled problem (all pointers are device pointers).
struct DevView {
  int nz, ncols, nnodes, npad, ncells, nelem, ninst, ntiles;
  int W, lsh;              // column block width (power of two, W * nz <= kTile) and log2 W
  int tile_threads;        // CTA size of the tile kernels: W * nz rounded up to whole warps
  int any_dirichlet;       // any prescribed node in the problem
  int sym;                 // matrix stored as its 14 upper stencil offsets (exactly symmetric)
  int minb;                // residual kernels: resident CTAs per SM they are built for (0 or 4)
  int grid_cap;            // CTAs of the tile kernels (0 = one per tile)
  int minb_k;              // Krylov matvecs (k_std_mv, k_cg_mv): the same, 0, 4, 6 or 8
  int grid_k;              // CTAs of the Krylov matvecs (0 = one per tile)
  int dry;                 // autotuner pass: Krylov matvecs run every tile, leave the state alone
  int solve2d;             // 2-D solve (shallow-shelf or L1L2): nz = 1, one 2-D element per cell
  int l1l2;                // L1L2: layer viscosities, 3-D velocity reconstructed after the loop
  int diva;                // DIVA: point viscosities carried between iterations, beta_eff, 3-D velocity each iteration
  int nl;                  // L1L2: layers of the velocity arrays (the model's nz - 1)
  unsigned long long* mv_nodes;  // [2] nodes through FP64 / FP32 Krylov matvecs (timing runs), or null
  const InstParams* inst;
  InstState* st;
  Counters* cnt;
  // columns
  const int* col_inst;     // [ncols]
  const int* col_nbr;      // [9][ncols], q = (jA+1)*3 + (iA+1); -1 = none
  const int* col_node;     // [ncols] node of (col, level 0); node (col, k) = col_node[col] + k * W
  const int* col_nbn;      // [9][ncols] col_node of each stencil neighbour; -1 = none
  const int* col_cells;    // [4][ncols], cells (i,j),(i+1,j),(i,j+1),(i+1,j+1)
  const int* col_ij;       // [2][ncols], halo'd Fortran vertex indices
  double* col_beta;        // [ncols] beta_internal (recomputed each Picard iteration with a sliding law)
  const double* col_slide; // [3][ncols] sliding law: f_ground and two per-vertex products, or null
  // nodes
  const double2* load;     // [nnodes] (loadu, loadv)
  const uint8_t* dmask;    // [nnodes] bit0 u prescribed, bit1 v prescribed
  // cells
  const int* cell_inst;    // [ncells]
  const int* cell_ij;      // [2][ncells] halo'd Fortran cell indices
  const int* cell_cols;    // [4][ncells] corner columns SW, SE, NE, NW (-1 = none)
  const double* cell_s;    // [4][ncells] stagusrf at the corners
  const double* cell_h;    // [4][ncells] stagthck at the corners
  double* cell_beta;       // [4][ncells] beta_internal at the corners (sliding law: 0 where no column)
  const double* flwafact;  // [nelem] (shallow-shelf: the column average per cell; L1L2: [ncells][nl])
  // L1L2 (null otherwise)
  const double* cell_flwa; // [ncells][nl] flow factor A
  const double* cell_thck; // [ncells] cell thickness
  const double* cell_ds;   // [2][4][ncells] surface gradient (x, y) at the corners
  const double* col_ds;    // [2][ncols] surface gradient at the column's vertex
  const double* col_h;     // [ncols] stagthck at the column's vertex
  double* lw;              // [4][nl][ncells] tau_parallel, w1, w2, w3 of the reconstruction
  double2* x3;             // [ncols][nl+1] reconstructed velocity (k = nl the bed); L1L2 and DIVA
  // DIVA (null otherwise)
  double* eq3;             // [ncells][4][nl] viscosity of each layer at each point (efvs_qp_3d)
  double* cell_omk;        // [ncells][nl+1] omega_k (Goldberg eq. 32, over H) per level
  double* cell_om;         // [ncells] omega (eq. 35, over H)
  const uint8_t* col_ipl;  // [ncols] ice-plus-land mask of the column's cells, bit q for cell q of col_cells
  double* col_somega;      // [ncols] omega staggered to the column
  double* col_beff;        // [ncols] beta_eff (the basal term of the 2-D system)
  double2* col_bt;         // [ncols] basal traction (btractx, btracty)
  // tiles: one per column block
  const int* tile_start;   // [ntiles] first node of the block
  const int* tile_end;     // [ntiles] tile_start + W * nz
  const int* tile_inst;    // [ntiles]
  const int* tile_ncols;   // [ntiles] columns in the block (the slots past them are holes)
  const int* tile_col0;    // [ntiles] first column of the block
  // assembly / matrix
  double* qp;              // [nelem*8*10]: f, Jinv(3x3) per quadrature point
  double* Ke;              // [nelem][4][8][8] element blocks (3-D element-centric assembly) or null
  double* efvs;            // [nelem]; L1L2 [ncells][nl]
  // FP64 matrix, (u,v) pairs: h = 0 the u-row (Auu, Auv), h = 1 the v-row
  // (Avu, Avv).  Full storage [2][27][npad]; symmetric storage [2][14][npad]
  // holds stencil offsets m = 13..26 (diagonal first), the lower half being
  // read from the neighbour's row.
  double2* A;
  // mixed: [14][npad] (uu, uv, vu, vv) of offsets 13..26 in FP32 (entry 0,
  // the diagonal block, unused by the matvec) and the diagonal block in
  // FP64 [2][npad], carrying the rounding of its row's off-diagonal
  // entries so that the row sums are those of the FP64 matrix
  float4* A32;
  double2* A32d;           // allocated right after A32 (one block of [16][npad] 16-byte elements)
  // L2 access-policy window carried by the PCG kernels' launches (host-side
  // launch setting; l2_bytes 0 = none)
  const void* l2_base;
  size_t l2_bytes;
  float l2_hit;
  double* badj;            // [4][npad] Dirichlet column moves per block
  double2* sia_f;          // [3][npad] SIA column preconditioner factors (a, beta, gamma), (u, v); or null
  // vectors (per node, (u,v) pairs)
  double2 *x, *b, *r, *z, *d0, *q, *Az, *Dinv, *usav;
  // reductions
  double* partials;        // [3][ntiles]
  unsigned* tile_counter;  // [ninst]
};

// Node of (col, k) in the blocked level-major layout.
BP_HD size_t node_of(const DevView& v, int col, int k) {
  return (size_t)v.col_node[col] + ((size_t)k << v.lsh);
}

// Column block width for nz levels: the largest power of two W with
// W * nz <= kTile.
BP_HD int block_width(int nz) {
  int w = 1;
  while (2 * w * nz <= kTile) w *= 2;
  return w;
}

// indxA_3d (glissade_velo_higher.F90:599-619), 0-based: iA fastest.
BP_HD int stencil_index(int iA, int jA, int kA) { return (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1); }

}  // namespace bp
