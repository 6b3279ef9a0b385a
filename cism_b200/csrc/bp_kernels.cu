// bp_kernels.cu -- sm_100a kernels of the Blatter-Pattyn solve.
//
// All node kernels walk tiles of at most kTile consecutive nodes (one tile per CTA
// iteration, grid-stride, so the same code runs as a one-shot grid or as a
// persistent grid).  A tile never spans two instances, so per-instance
// reductions are: block reduce -> per-tile partial -> the last CTA of the
// instance (atomic ticket) sums the partials in tile order and runs the
// scalar update (alpha, beta, convergence) on the device.  The result is
// bitwise reproducible run to run and needs no host round trip.
#include <cstdio>

#include "bp_body.h"
#include "bp_b200.h"
#include "bp_kernels.h"

#include <cstdlib>

namespace bp {

__constant__ RefTables c_T;

// ---------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------
template <int NV, bool MAX0>
__device__ __forceinline__ void block_reduce(double (&val)[NV], double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double x = val[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, o);
      x = (MAX0 && i == 0) ? fmax(x, y) : x + y;
    }
    if (lane == 0) sm[i * 32 + warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = lane < nw ? sm[i * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, x, o);
        x = (MAX0 && i == 0) ? fmax(x, y) : x + y;
      }
      val[i] = x;
    }
  }
  __syncthreads();
}

// Reduce NV values of this tile; the last tile of the instance sums all
// tile partials of the instance in tile order and calls fin(inst, sums).
template <int NV, bool MAX0, typename Fin>
__device__ __forceinline__ void tile_finish(const DevView& v, int t, int inst,
                                            double (&val)[NV], Fin fin) {
  __shared__ double sm[NV * 32];
  __shared__ int last;
  block_reduce<NV, MAX0>(val, sm);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v.partials[(size_t)i * v.ntiles + t] = val[i];
    __threadfence();
    const InstParams& ip = v.inst[inst];
    const unsigned ntl = (unsigned)(ip.tile_end - ip.tile_begin);
    const unsigned prev = atomicAdd(&v.tile_counter[inst], 1u);
    last = (prev == ntl - 1) ? 1 : 0;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    const InstParams& ip = v.inst[inst];
    double s[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) s[i] = 0.0;
    for (int tt = ip.tile_begin + threadIdx.x; tt < ip.tile_end; tt += blockDim.x)
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const double p = __ldcg(v.partials + (size_t)i * v.ntiles + tt);
        s[i] = (MAX0 && i == 0) ? fmax(s[i], p) : s[i] + p;
      }
    block_reduce<NV, MAX0>(s, sm);
    if (threadIdx.x == 0) {
      v.tile_counter[inst] = 0;
      fin(inst, s);
      __threadfence();
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void pcg_stop(const DevView& v, InstState& S, bool converged) {
  S.pcg_active = 0;
  S.pcg_converged = converged ? 1 : 0;
  S.pcg_iters_last = S.pcg_iter;
  S.pcg_iters_total += S.pcg_iter;
  atomicSub(&v.cnt->pcg_active, 1);
}

__device__ __forceinline__ void fail(const DevView& v, InstState& S, int code) {
  if (S.status == BP_OK || S.status == BP_WARN_PCG_NOT_CONVERGED) S.status = code;
  if (S.pcg_active) pcg_stop(v, S, false);
  if (S.refine_active) {
    S.refine_active = 0;
    atomicSub(&v.cnt->refine_active, 1);
  }
  if (S.picard_active) {
    S.picard_active = 0;
    atomicSub(&v.cnt->picard_active, 1);
  }
}

__device__ __forceinline__ bool is_nan(double x) { return x != x; }

struct TileRange {
  int inst, n0, nend, ncols, col0;
};

// Programmatic dependent launch: the PCG kernels are launched so that the
// next one may be scheduled while its predecessor drains; each calls
// pdl_wait() (which returns once the predecessor grid has completed and its
// writes are visible) before it reads anything, in every CTA, so a grid
// also completes only after its predecessor.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_next() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ TileRange tile_range(const DevView& v, int t) {
  TileRange r;
  r.inst = v.tile_inst[t];
  r.n0 = v.tile_start[t];
  r.nend = v.tile_end[t];
  r.ncols = v.tile_ncols[t];
  r.col0 = v.tile_col0[t];
  return r;
}

// Thread i of a tile's CTA owns node n0 + i: level i >> lsh, column col0 +
// (i & (W-1)); the slots past the block's columns are holes.
__device__ __forceinline__ bool tile_mine(const DevView& v, const TileRange& R, int i) {
  return R.n0 + i < R.nend && (i & (v.W - 1)) < R.ncols;
}
__device__ __forceinline__ int tile_col(const DevView& v, const TileRange& R, int i) {
  return R.col0 + (i & (v.W - 1));
}
__device__ __forceinline__ int tile_k(const DevView& v, int i) { return i >> v.lsh; }

// ---------------------------------------------------------------------
// Picard iteration start (one CTA): counter, reset of the PCG state.
// ---------------------------------------------------------------------
__global__ void k_picard_begin(DevView v) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int i = threadIdx.x; i < v.ninst; i += blockDim.x) {
    InstState& S = v.st[i];
    if (!S.picard_active) continue;
    S.picard_iter += 1;
    S.nonzero = 0;
    S.pcg_active = 1;
    S.pcg_iter = 1;
    S.pcg_converged = 0;
    S.rz = 1.0;
    S.rz_old = 1.0;
    S.alpha = 0.0;
    S.beta = 0.0;
    S.err = -1.0;
    S.refine_steps = 0;
    S.refine_active = 1;
    S.inner_iter = 0;
    S.pcg_iters_last = 0;
    S.krylov_fp64 = 0;
    S.need_true = 0;
    S.restart = 0;
    S.last_true_iter = 0;
    S.r_true = 0.0;
    ++mine;
  }
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    v.cnt->pcg_active = cnt;
    v.cnt->refine_active = cnt;
  }
}

// calcbeta with a velocity-dependent law at the start of a Picard iteration
// (glissade_velo_higher.F90:2502-2517): beta of every column of an active
// instance from its basal velocity x(nz-1).  An invalid beta (negative or
// NaN, glissade_basal_traction.F90:570-582) marks the instance; k_rhs ends
// it with BP_ERR_BAD_BETA before its linear solve.
__global__ void __launch_bounds__(kTile) k_slide_beta(DevView v) {
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < v.ncols; col += gridDim.x * blockDim.x) {
    const int inst = v.col_inst[col];
    const InstParams& ip = v.inst[inst];
    InstState& S = v.st[inst];
    if (!S.picard_active || ip.slide.law == 0) continue;
    const size_t nc = (size_t)v.ncols;
    // the basal velocity: DIVA's 3-D one (:2240-2243), else the bed node
    const double2 ub = v.diva ? v.x3[(size_t)col * (v.nl + 1) + v.nl] : v.x[node_of(v, col, v.nz - 1)];
    const double beta = slide_beta(ip.slide, v.col_slide[col], v.col_slide[nc + col],
                                   v.col_slide[2 * nc + col], ub.x, ub.y);
    if (!(beta >= 0.0) && (S.status == BP_OK || S.status == BP_WARN_PCG_NOT_CONVERGED))
      S.status = BP_ERR_BAD_BETA;
    v.col_beta[col] = beta;
  }
}

// Corner betas of the bed faces for the standard basal assembly
// (basal_sliding_bc :8234-8363) after k_slide_beta: the corner's column,
// or 0 where the corner has no column (a vertex outside an outflow domain,
// zeroed by the staggered halo update).
__global__ void __launch_bounds__(kTile) k_cell_beta(DevView v) {
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < v.ncells; cell += gridDim.x * blockDim.x) {
    const int inst = v.cell_inst[cell];
    if (!v.st[inst].picard_active || v.inst[inst].slide.law == 0) continue;
    for (int q = 0; q < 4; ++q) {
      const int col = v.cell_cols[(size_t)q * v.ncells + cell];
      v.cell_beta[(size_t)q * v.ncells + cell] = col >= 0 ? v.col_beta[col] : 0.0;
    }
  }
}

__global__ void __launch_bounds__(kTile) k_save_usav(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].picard_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (tile_mine(v, R, threadIdx.x)) v.usav[n] = v.x[n];
  }
}

// ---------------------------------------------------------------------
// Assembly pass 1: thread = (element, quadrature point).
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_asm_qp(DevView v) {
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = (int)(gtid >> 3), p = (int)(gtid & 7);
  bool valid = e < v.nelem;
  int inst = 0;
  if (valid) {
    inst = v.cell_inst[e / (v.nz - 1)];
    valid = v.st[inst].picard_active != 0;
  }
  const unsigned mask = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  double out[10], eq = 0.0;
  const bool ok = qp_element_point(v, c_T, e, p, out, &eq);
  if (!ok) {
    atomicExch(&v.st[inst].status, BP_ERR_SINGULAR_JAC);
    eq = 0.0;
#pragma unroll
    for (int i = 0; i < 10; ++i) out[i] = 0.0;
  }
  double2* dst = reinterpret_cast<double2*>(v.qp + ((size_t)e * 8 + p) * 10);
#pragma unroll
  for (int i = 0; i < 5; ++i) dst[i] = make_double2(out[2 * i], out[2 * i + 1]);
  // element average of the quadrature-point viscosity, in point order
  const int lane0 = (threadIdx.x & 31) & ~7;
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += __shfl_sync(mask, eq, lane0 + q);
  if (p == 0) v.efvs[e] = s / 8.0;
}

// Pass 1 of the shallow-shelf assembly: one thread per (active cell, 2-D
// point), the cell's viscosity the mean of its 4 points (:5539-5545).
// LAYERS: the L1L2 and DIVA solves, with a viscosity per layer (kept in
// a per-thread array the shallow-shelf instance does without).
template <bool LAYERS>
__global__ void __launch_bounds__(256) k_asm2_qp(DevView v) {
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(gtid >> 2), p = (int)(gtid & 3);
  bool valid = c < v.ncells;
  int inst = 0;
  if (valid) {
    inst = v.cell_inst[c];
    valid = v.st[inst].picard_active != 0;
  }
  const unsigned mask = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  double out[5], eq = 0.0, ek[LAYERS ? kNzMax - 1 : 1];
  const bool ok = qp2_element_point(v, c_T, c, p, out, &eq, LAYERS ? ek : nullptr);
  if (!ok) {
    atomicExch(&v.st[inst].status, BP_ERR_SINGULAR_JAC);
    eq = 0.0;
    for (int i = 0; i < 5; ++i) out[i] = 0.0;
  }
  double* dst = v.qp + ((size_t)c * 8 + p) * 10;
  for (int i = 0; i < 5; ++i) dst[i] = out[i];
  const int lane0 = (threadIdx.x & 31) & ~3;
  if (LAYERS) {  // efvs(k) = the mean of the layer's point values (:5565-5572)
    for (int k = 0; k < v.nl; ++k) {
      const double e = ok ? ek[k] : 0.0;
      double sum = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) sum += __shfl_sync(mask, e, lane0 + q);
      if (p == 0) v.efvs[(size_t)c * v.nl + k] = sum / 4.0;
    }
    return;
  }
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) sum += __shfl_sync(mask, eq, lane0 + q);
  if (p == 0) v.efvs[c] = sum / 4.0;
}

// L1L2 3-D velocity after the Picard loop (compute_3d_velocity_L1L2,
// glissade_velo_higher.F90:5834-6356): the cell pass (l1l2_cell), then
// one thread per column integrates from the bed up (l1l2_column).  Run
// once per solve; bounded by the nl * 4 cell values each column reads.
__global__ void __launch_bounds__(256) k_l1l2_cells(DevView v) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < v.ncells) l1l2_cell(v, c);
}

__global__ void __launch_bounds__(256) k_l1l2_columns(DevView v) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col < v.ncols) l1l2_column(v, col);
}

// DIVA, every Picard iteration of an active instance: after assembly pass
// 1 the cells' omega integrals (k_diva_cells), beta_eff at the columns
// (k_diva_beta) and at the bed-face corners for the standard basal
// assembly (k_diva_cell_beta); after the linear solve the traction and
// the 3-D velocity (k_diva_velocity).
__global__ void __launch_bounds__(256) k_diva_cells(DevView v) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < v.ncells && v.st[v.cell_inst[c]].picard_active) diva_cell_integrals(v, c);
}

__global__ void __launch_bounds__(256) k_diva_beta(DevView v) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col < v.ncols && v.st[v.col_inst[col]].picard_active) diva_column_beta(v, col);
}

__global__ void __launch_bounds__(256) k_diva_cell_beta(DevView v) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= v.ncells || !v.st[v.cell_inst[cell]].picard_active) return;
  for (int q = 0; q < 4; ++q) {
    const int col = v.cell_cols[(size_t)q * v.ncells + cell];
    v.cell_beta[(size_t)q * v.ncells + cell] = col >= 0 ? v.col_beff[col] : 0.0;
  }
}

__global__ void __launch_bounds__(256) k_diva_velocity(DevView v) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col < v.ncols && v.st[v.col_inst[col]].picard_active) diva_column_velocity(v, col);
}

// ---------------------------------------------------------------------
// Assembly pass 2 + basal BC + Dirichlet BC: thread = (block B, node).
// ---------------------------------------------------------------------
enum { ASM_ROWS = 0, ASM_GATHER = 1, ASM_2D = 2 };

// Element-centric pass 2a: thread = (element, corner nr); the corner's rows
// of the element's four blocks (element_row_blocks) into Ke, the eight
// threads of an element writing 64 consecutive doubles per block.
__global__ void __launch_bounds__(256, 2) k_asm_elem(DevView v) {
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = (int)(gtid >> 3), nr = (int)(gtid & 7);
  if (e >= v.nelem) return;
  if (!v.st[v.cell_inst[e / (v.nz - 1)]].picard_active) return;
  double K[32];
  element_row_blocks(c_T, v.qp + (size_t)e * 80, nr, K);
  double2* out = reinterpret_cast<double2*>(v.Ke + (size_t)e * 256 + nr * 8);
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int i = 0; i < 4; ++i) out[b * 32 + i] = make_double2(K[b * 8 + 2 * i], K[b * 8 + 2 * i + 1]);
}
template <int B, int MODE>
__device__ __forceinline__ bool asm_row(const DevView& v, int n, int col, int k) {
  double acc[27];
  if (MODE == ASM_2D) row_assemble2<B>(v, c_T, col, acc);
  else if (MODE == ASM_GATHER) row_gather<B>(v, v.Ke, col, k, acc);
  else row_assemble<B>(v, c_T, col, k, acc);
  row_basal<B>(v, c_T, col, k, acc);
  const double adj = row_dirichlet<B>(v, col, k, acc);
  bool nz = false;
  double* Ad = reinterpret_cast<double*>(v.A);
  const size_t np = (size_t)v.npad;
  const int h = B >> 1, comp = B & 1;
#pragma unroll
  for (int m = 0; m < 27; ++m) {
    nz |= (acc[m] != 0.0);
    if (v.sym) {
      if (m >= 13) Ad[(((size_t)(h * 14 + m - 13)) * np + n) * 2 + comp] = acc[m];
    } else {
      Ad[(((size_t)(h * 27 + m)) * np + n) * 2 + comp] = acc[m];
    }
  }
  v.badj[(size_t)B * np + n] = adj;
  return nz;
}

// MODE: ASM_ROWS (3-D, each row integrates its incident elements),
// ASM_GATHER (3-D, each row sums the element rows k_asm_elem stored) or
// ASM_2D (the rows of the 2-D solves: shallow-shelf, L1L2; nz = 1).
template <int MODE>
__global__ void __launch_bounds__(kTile) k_asm_rows(DevView v) {
  const int B = blockIdx.y;
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].picard_active) continue;
    const int n = R.n0 + threadIdx.x;
    int nzl = 0;
    if (tile_mine(v, R, threadIdx.x)) {
      const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
      switch (B) {
        case 0: nzl = asm_row<0, MODE>(v, n, col, k); break;
        case 1: nzl = asm_row<1, MODE>(v, n, col, k); break;
        case 2: nzl = asm_row<2, MODE>(v, n, col, k); break;
        default: nzl = asm_row<3, MODE>(v, n, col, k); break;
      }
    }
    if (__syncthreads_or(nzl) && threadIdx.x == 0) atomicOr(&v.st[R.inst].nonzero, 1);
  }
}

// ---------------------------------------------------------------------
// Right-hand side (load + Dirichlet moves), preconditioner, (b,b).
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) k_rhs(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].picard_active) continue;
    const InstParams& ip = v.inst[R.inst];
    const int n = R.n0 + threadIdx.x;
    double part[1] = {0.0};
    if (tile_mine(v, R, threadIdx.x)) {
      const size_t np = (size_t)v.npad;
      const uint8_t dm = v.dmask[n];
      const double2 ld = v.load[n];
      const double2 xn = v.x[n];
      double bu = ld.x - v.badj[0 * np + n] - v.badj[1 * np + n];
      double bv = ld.y - v.badj[2 * np + n] - v.badj[3 * np + n];
      if (dm & 1) bu = xn.x;
      if (dm & 2) bv = xn.y;
      v.b[n] = make_double2(bu, bv);
      double2 di = make_double2(1.0, 1.0);
      if (ip.precond == 1) {
        const double du = diag_u(v, n), dv = diag_v(v, n);
        di.x = du != 0.0 ? 1.0 / du : 0.0;
        di.y = dv != 0.0 ? 1.0 / dv : 0.0;
      }
      v.Dinv[n] = di;
      part[0] = bu * bu + bv * bv;
    }
    tile_finish<1, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      InstState& S = v.st[inst];
      S.bb = s[0];
      S.L2_rhs = sqrt(s[0]);
      if (S.status == BP_ERR_SINGULAR_JAC || S.status == BP_ERR_BAD_BETA) {
        fail(v, S, S.status);
      } else if (!S.nonzero) {
        S.status = BP_ZERO_MATRIX;
        S.zero_x = 1;
        fail(v, S, BP_ZERO_MATRIX);
      } else if (v.solve2d && !v.diva && v.inst[inst].which_babc == 6) {
        // 2-D solve on a no-slip bed: the 2-D velocity is zero and nothing is solved
        // (glissade_velo_higher.F90:3227-3240)
        S.frozen = 1;
        S.L2_norm = 0.0;
        S.L2_rel = 0.0;
        S.pcg_iter = 0;
        pcg_stop(v, S, true);
        if (S.refine_active) {
          S.refine_active = 0;
          atomicSub(&v.cnt->refine_active, 1);
        }
      }
    });
  }
}

// ---------------------------------------------------------------------
// SIA column preconditioner on a tile of whole columns: every thread puts
// its node's r and its node's factors (a, beta, gamma for u and v) into
// shared memory, one thread per (column, component) runs the two Thomas
// sweeps from there (sia_sweeps), every thread takes back its z.  The
// sweeps are a chain of dependent steps; with the factors staged by
// coalesced loads beforehand, no step of the chain waits on global memory.
// Called by all threads of the CTA (uniform per tile).
// ---------------------------------------------------------------------
struct SiaTile {
  double s[2 * kTile], a[2 * kTile], b[2 * kTile], g[2 * kTile];
};

__device__ __forceinline__ double2 sia_tile(const DevView& v, const TileRange& R, double2 r) {
  __shared__ SiaTile T;
  const int i = threadIdx.x, nz = v.nz;
  const bool mine = tile_mine(v, R, i);
  // shared memory holds the tile column by column: j = c * nz + k
  const int k = tile_k(v, i), j = (i & (v.W - 1)) * nz + k;
  if (mine) {
    const size_t n = (size_t)R.n0 + i, np = (size_t)v.npad;
    const double2 fa = v.sia_f[n], fb = v.sia_f[np + n], fg = v.sia_f[2 * np + n];
    T.s[2 * j] = r.x;
    T.s[2 * j + 1] = r.y;
    T.a[2 * j] = fa.x;
    T.a[2 * j + 1] = fa.y;
    T.b[2 * j] = fb.x;
    T.b[2 * j + 1] = fb.y;
    T.g[2 * j] = fg.x;
    T.g[2 * j + 1] = fg.y;
  }
  __syncthreads();
  if (i < 2 * R.ncols) {
    const int c = i >> 1, h = i & 1, o = 2 * c * nz + h;
    sia_sweeps(
        nz, [&](int kk) { return SiaFac{T.a[o + 2 * kk], T.b[o + 2 * kk], T.g[o + 2 * kk]}; }, &T.s[o], 2);
  }
  __syncthreads();
  const double2 z = mine ? make_double2(T.s[2 * j], T.s[2 * j + 1]) : make_double2(0.0, 0.0);
  __syncthreads();  // T is reused by the CTA's next tile
  return z;
}

// z = M^-1 r for the instance's preconditioner (diagonal or none: D^-1
// from k_rhs / k_dinv; SIA: column solves).  Called by all threads.
__device__ __forceinline__ double2 precondition(const DevView& v, const TileRange& R, bool mine, size_t n,
                                                double2 r) {
  if (v.inst[R.inst].precond == 2) return sia_tile(v, R, r);
  if (!mine) return make_double2(0.0, 0.0);
  const double2 di = v.Dinv[n];
  return make_double2(r.x * di.x, r.y * di.y);
}

// ---------------------------------------------------------------------
// PCG kernels.  Every Krylov matvec reads one stored source vector (d for
// the standard PCG, z = D^-1 r for Chronopoulos-Gear, x for residuals), so
// each matvec is a plain y = A s with its dot products fused in.  Storage
// variants: full FP64 rows, symmetric FP64, symmetric FP32 (Krylov matvecs
// of the mixed path; residuals always use the FP64 matrix).
// ---------------------------------------------------------------------
enum { ST_FULL = 0, ST_SYM = 1, ST_SYM32 = 2 };

struct SrcX {
  const double2* x;
  __device__ double2 operator()(size_t m) const { return x[m]; }
};

template <int STORE>
__device__ __forceinline__ double2 mv_row(const DevView& v, int col, int k, size_t n,
                                          const double2* s) {
  const SrcX src{s};
  if (STORE == ST_FULL) return matvec_row(v, v.A, col, k, n, src);
  if (STORE == ST_SYM) return matvec_row_sym(v, v.A, col, k, n, src);
  return matvec_row_sym32(v, v.A32, col, k, n, src);
}

// Mixed precision (iterative refinement): the Krylov iteration runs on the
// FP32 matrix with FP64 vectors and reductions; the FP64 residual b - A x
// replaces the recurrence residual only once the latter has fallen by
// inner_tol since the last replacement (or below the final tolerance, or
// after 500 iterations), and each replacement restarts the Krylov process,
// so every cycle is a clean conjugate-gradient solve of A32 e = r.  Called
// after iteration pcg_iter; replacements follow iterations that are
// multiples of ncheck.
__device__ __forceinline__ void refine_request(const InstParams& ip, InstState& S, double rr) {
  if (S.pcg_iter % ip.ncheck != 0) return;
  const double rn = sqrt(rr);
  if (rn < ip.inner_tol * S.r_true || rn < 0.5 * ip.pcg_tol * S.L2_rhs ||
      S.pcg_iter - S.last_true_iter >= 500)
    S.need_true = 1;
}

// r = b - A x with the FP64 matrix; z = D^-1 r stored; (r,z) and (r,r).
// MV_INIT starts a linear solve (also compute_residual_vector_3d's norms);
// MV_CHECK is the every-ncheck true residual (pcg:478-536, 1542-1597);
// MV_REFINE the mixed-precision refinement step, for instances that
// requested it.
template <int MODE, int STORE, int MINB>
__global__ void __launch_bounds__(kTile, MINB) k_resid(DevView v) {
  pdl_wait();
  pdl_launch_next();
  constexpr int ST64 = STORE == ST_SYM32 ? ST_SYM : STORE;
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S0 = v.st[R.inst];
    if (!S0.pcg_active || (MODE == MV_REFINE && !S0.need_true)) continue;
    const int n = R.n0 + threadIdx.x;
    const bool mine = tile_mine(v, R, threadIdx.x);
    double part[2] = {0.0, 0.0};
    double2 r = make_double2(0.0, 0.0);
    if (mine) {
      const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
      const double2 y = mv_row<ST64>(v, col, k, n, v.x);
      const double2 b = v.b[n];
      r = make_double2(b.x - y.x, b.y - y.y);
    }
    const double2 z = precondition(v, R, mine, n, r);
    if (mine) {
      v.r[n] = r;
      v.z[n] = z;
      part[0] = r.x * z.x + r.y * z.y;
      part[1] = r.x * r.x + r.y * r.y;
    }
    tile_finish<2, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      InstState& S = v.st[inst];
      const InstParams& ip = v.inst[inst];
      const double rt = sqrt(s[1]);
      if (MODE == MV_INIT) {
        S.L2_norm = rt;
        S.L2_rel = S.L2_rhs > 0.0 ? S.L2_norm / S.L2_rhs : 0.0;
        S.r_true = rt;
        S.last_true_iter = S.pcg_iter;
      } else {
        S.err = rt / S.L2_rhs;
        S.refine_steps_total += 1;
        if (MODE == MV_REFINE) {
          S.need_true = 0;
          S.last_true_iter = S.pcg_iter;
        }
        if (S.err < ip.pcg_tol) { pcg_stop(v, S, true); return; }
        if (S.pcg_iter >= ip.pcg_maxiters) { pcg_stop(v, S, false); return; }
        if (MODE == MV_REFINE) {
          // a cycle that did not halve the residual: the FP32 operator is
          // too coarse for this system, finish with the FP64 matrix
          if (rt > 0.5 * S.r_true) S.krylov_fp64 = 1;
          S.r_true = rt;
        }
      }
      if (ip.variant != 3) {  // standard PCG: eta1 of the next iteration
        if (is_nan(s[0])) { fail(v, S, BP_ERR_NAN); return; }
        S.beta = MODE == MV_REFINE ? 0.0 : s[0] / S.rz;  // refinement restarts: d = z
        S.rz = s[0];
        if (MODE == MV_CHECK) S.pcg_iter += 1;
      } else if (MODE == MV_REFINE) {
        S.restart = 1;
      }
    });
  }
}

// Krylov matvec of the mixed path: FP32 matrix unless the instance's
// refinement stalled (krylov_fp64), FP64 then.  In timing runs the nodes
// through each precision are counted, to turn the measured time into bytes.
// The FP64 Krylov matvec of an instance whose FP32 refinement stalled,
// out of line: inlined, its registers would count against every launch of
// the FP32 kernel, which is sized to fit 32 registers per thread.
struct MvGeom {
  int nz, ncols, npad, lsh;
  const int* col_nbn;
};
__device__ __noinline__ double2 mv_row_sym64_call(MvGeom g, const double2* A, int col, int k, size_t n,
                                                  const double2* s) {
  return matvec_row_sym(g, A, col, k, n, SrcX{s});
}

template <int STORE>
__device__ __forceinline__ double2 krylov_row(const DevView& v, const InstState& S, int col, int k,
                                              size_t n, const double2* s) {
  if (STORE == ST_SYM32 && S.krylov_fp64)
    return mv_row_sym64_call(MvGeom{v.nz, v.ncols, v.npad, v.lsh, v.col_nbn}, v.A, col, k, n, s);
  return mv_row<STORE>(v, col, k, n, s);
}

template <int STORE>
__device__ __forceinline__ void count_tile(const DevView& v, const InstState& S, const TileRange& R) {
  if (v.mv_nodes && !v.dry && threadIdx.x == 0) {
    const bool f32 = STORE == ST_SYM32 && !S.krylov_fp64;
    atomicAdd(&v.mv_nodes[f32 ? 1 : 0], (unsigned long long)R.ncols * v.nz);
  }
}

// alpha = eta1 / (d, q) of the standard PCG (pcg:426-463).
__device__ __forceinline__ void std_mv_fin(const DevView& v, int inst, const double* s) {
  if (v.dry) return;
  InstState& S = v.st[inst];
  const double alpha = S.rz / s[0];
  if (is_nan(alpha)) { fail(v, S, BP_ERR_NAN); return; }
  S.alpha = alpha;
}

// The Chronopoulos-Gear scalar recurrences from (r,z), (Az,z), (r,r)
// (pcg:1461-1512); FIRST: the first pass (pcg:1304-1405).
template <bool FIRST>
__device__ __forceinline__ void cg_mv_fin(const DevView& v, int inst, const double* s) {
  if (v.dry) return;
  InstState& S = v.st[inst];
  if (FIRST) {
    S.rz_old = s[0];
    S.sigma = s[1];
    const double alpha = s[0] / s[1];
    if (is_nan(alpha)) { fail(v, S, BP_ERR_NAN); return; }
    S.alpha = alpha;
    return;
  }
  const InstParams& ip = v.inst[inst];
  S.pcg_iter += 1;
  if (S.pcg_iter > ip.pcg_maxiters) {
    S.pcg_iter = ip.pcg_maxiters;
    pcg_stop(v, S, false);
    return;
  }
  const double rho = s[0], delta = s[1];
  double beta, sigma;
  if (S.restart) {  // after a refinement: d = z, q = A z (the first pass)
    beta = 0.0;
    sigma = delta;
    S.restart = 0;
  } else {
    beta = rho / S.rz_old;
    sigma = delta - beta * rho / S.alpha;
  }
  const double alpha = rho / sigma;
  S.rz_old = rho;
  S.beta = beta;
  S.sigma = sigma;
  if (is_nan(alpha)) { fail(v, S, BP_ERR_NAN); return; }
  S.alpha = alpha;
  if (v.A32) refine_request(ip, S, s[2]);
}

// Standard PCG: q = A d; (d, q); alpha = eta1 / (d, q)   (pcg:426-463).
// In the autotuner's dry pass (v.dry) the Krylov matvecs run on every tile
// and skip the scalar tail, so timing them changes no instance state.
template <int STORE, int MINB>
__global__ void __launch_bounds__(kTile, MINB) k_std_mv(DevView v) {
  pdl_wait();
  pdl_launch_next();
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S0 = v.st[R.inst];
    if (!S0.pcg_active && !v.dry) continue;
    count_tile<STORE>(v, S0, R);
    const int n = R.n0 + threadIdx.x;
    double part[1] = {0.0};
    if (tile_mine(v, R, threadIdx.x)) {
      const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
      const double2 y = krylov_row<STORE>(v, S0, col, k, n, v.d0);
      const double2 d = v.d0[n];
      v.q[n] = y;
      part[0] = d.x * y.x + d.y * y.y;
    }
    tile_finish<1, false>(v, t, R.inst, part, [&](int inst, const double* s) { std_mv_fin(v, inst, s); });
  }
}

// x += alpha d; r -= alpha q; z = D^-1 r; (r, z) -> beta  (pcg:347-407, 468-472).
// On check iterations only x is updated (r is recomputed from b - A x).
template <bool CHECK>
__global__ void __launch_bounds__(kTile) k_std_update(DevView v) {
  pdl_wait();
  pdl_launch_next();
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    const double alpha = S.alpha;
    const bool mine = tile_mine(v, R, threadIdx.x);
    double part[2] = {0.0, 0.0};
    double2 r = make_double2(0.0, 0.0);
    if (mine) {
      const double2 d = v.d0[n];
      double2 x = v.x[n];
      x.x = x.x + alpha * d.x;
      x.y = x.y + alpha * d.y;
      v.x[n] = x;
      if (!CHECK) {
        const double2 q = v.q[n];
        r = v.r[n];
        r.x = r.x - alpha * q.x;
        r.y = r.y - alpha * q.y;
        v.r[n] = r;
      }
    }
    if (!CHECK) {
      const double2 z = precondition(v, R, mine, n, r);
      if (mine) {
        v.z[n] = z;
        part[0] = r.x * z.x + r.y * z.y;
        part[1] = r.x * r.x + r.y * r.y;
      }
    }
    if (!CHECK) {
      tile_finish<2, false>(v, t, R.inst, part, [&](int inst, const double* s) {
        InstState& S2 = v.st[inst];
        const InstParams& ip = v.inst[inst];
        if (S2.pcg_iter >= ip.pcg_maxiters) { pcg_stop(v, S2, false); return; }
        if (is_nan(s[0])) { fail(v, S2, BP_ERR_NAN); return; }
        S2.beta = s[0] / S2.rz;
        S2.rz = s[0];
        if (v.A32) refine_request(ip, S2, s[1]);
        S2.pcg_iter += 1;
      });
    }
  }
}

// d = z + beta d; d = z at the first iteration (pcg:403-407).
__global__ void __launch_bounds__(kTile) k_std_dir(DevView v) {
  pdl_wait();
  pdl_launch_next();
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (!tile_mine(v, R, threadIdx.x)) continue;
    const double2 z = v.z[n];
    if (S.pcg_iter == 1) {
      v.d0[n] = z;
    } else {
      const double beta = S.beta;
      const double2 d = v.d0[n];
      v.d0[n] = make_double2(z.x + beta * d.x, z.y + beta * d.y);
    }
  }
}

// Chronopoulos-Gear matvec Az = A z with (r,z), (Az,z) and the scalar
// recurrences (pcg:1461-1512).  FIRST: the first pass (pcg:1304-1405),
// which also sets d = z, q = A d.
template <bool FIRST, int STORE, int MINB>
__global__ void __launch_bounds__(kTile, MINB) k_cg_mv(DevView v) {
  pdl_wait();
  pdl_launch_next();
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S0 = v.st[R.inst];
    if (!S0.pcg_active && !v.dry) continue;
    count_tile<STORE>(v, S0, R);
    const int n = R.n0 + threadIdx.x;
    double part[3] = {0.0, 0.0, 0.0};
    if (tile_mine(v, R, threadIdx.x)) {
      const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
      const double2 y = krylov_row<STORE>(v, S0, col, k, n, v.z);
      const double2 z = v.z[n], r = v.r[n];
      if (FIRST) {
        v.d0[n] = z;
        v.q[n] = y;
      } else {
        v.Az[n] = y;
      }
      part[0] = r.x * z.x + r.y * z.y;
      part[1] = y.x * z.x + y.y * z.y;
      part[2] = r.x * r.x + r.y * r.y;
    }
    tile_finish<3, false>(v, t, R.inst, part, [&](int inst, const double* s) { cg_mv_fin<FIRST>(v, inst, s); });
  }
}

// Chronopoulos-Gear first-pass update: x += alpha d; r -= alpha q; z = D^-1 r.
__global__ void __launch_bounds__(kTile) k_cg_first_update(DevView v) {
  pdl_wait();
  pdl_launch_next();
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    const bool mine = tile_mine(v, R, threadIdx.x);
    const double alpha = S.alpha;
    double2 r = make_double2(0.0, 0.0);
    if (mine) {
      const double2 d = v.d0[n], q = v.q[n];
      double2 x = v.x[n];
      r = v.r[n];
      x.x = x.x + alpha * d.x; x.y = x.y + alpha * d.y;
      r.x = r.x - alpha * q.x; r.y = r.y - alpha * q.y;
      v.x[n] = x;
      v.r[n] = r;
    }
    const double2 z = precondition(v, R, mine, n, r);
    if (mine) v.z[n] = z;
  }
}

// Chronopoulos-Gear loop update (pcg:1519-1534): d = z + beta d;
// q = Az + beta q; x += alpha d; r -= alpha q; z = D^-1 r for the next
// iteration (skipped on check iterations, where r and z come from b - A x).
template <bool CHECK>
__global__ void __launch_bounds__(kTile) k_cg_update(DevView v) {
  pdl_wait();
  pdl_launch_next();
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    const bool mine = tile_mine(v, R, threadIdx.x);
    const bool keep_r = !CHECK && !S.need_true;  // a refinement recomputes r and z
    const double alpha = S.alpha, beta = S.beta;
    double2 r = make_double2(0.0, 0.0);
    if (mine) {
      const double2 z = v.z[n], az = v.Az[n];
      double2 d = v.d0[n], q = v.q[n], x = v.x[n];
      d.x = z.x + beta * d.x; d.y = z.y + beta * d.y;
      q.x = az.x + beta * q.x; q.y = az.y + beta * q.y;
      x.x = x.x + alpha * d.x; x.y = x.y + alpha * d.y;
      v.d0[n] = d;
      v.q[n] = q;
      v.x[n] = x;
      if (keep_r) {
        r = v.r[n];
        r.x = r.x - alpha * q.x;
        r.y = r.y - alpha * q.y;
        v.r[n] = r;
      }
    }
    if (keep_r) {
      const double2 z = precondition(v, R, mine, n, r);
      if (mine) v.z[n] = z;
    }
  }
}

// ---------------------------------------------------------------------
// Picard convergence: compute_residual_velocity_3d (:9111-9234).
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) k_picard_check(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    InstState& S = v.st[R.inst];
    const InstParams& ip = v.inst[R.inst];
    const int n = R.n0 + threadIdx.x;
    const bool mine = tile_mine(v, R, threadIdx.x);
    if (S.zero_x) {
      if (mine) v.x[n] = make_double2(0.0, 0.0);
      continue;
    }
    if (!S.picard_active) continue;
    const bool meanu = ip.which_resid == 2;
    // the 2-D criterion has no bed layer to leave out (:9238-9351)
    const bool nobed = !v.solve2d && (ip.which_resid == 1 || meanu);
    double part[2] = {0.0, 0.0};
    if (mine) {
      if (S.frozen) v.x[n] = make_double2(0.0, 0.0);  // 2-D solve on a no-slip bed
      const int k = tile_k(v, threadIdx.x);
      if (!(nobed && k == v.nz - 1)) {
        const double2 x = v.x[n], o = v.usav[n];
        const double speed = sqrt(x.x * x.x + x.y * x.y);
        if (speed != 0.0) {
          const double old = sqrt(o.x * o.x + o.y * o.y);
          part[0] = fabs((old - speed) / speed);
          part[1] = 1.0;
        }
      }
    }
    auto fin = [&](int inst, const double* s) {
      InstState& S2 = v.st[inst];
      const InstParams& ip2 = v.inst[inst];
      const bool mean2 = ip2.which_resid == 2;
      S2.resid_velo = mean2 ? (s[1] > 0.0 ? s[0] / s[1] : 0.0) : s[0];
      double crit, target;
      if (ip2.which_resid == 3) { crit = S2.L2_norm; target = 1.0e-4; }
      else if (ip2.which_resid == 4) { crit = S2.L2_rel; target = 1.0e-7; }
      else { crit = S2.resid_velo; target = 1.0e-4; }
      const bool done = !(crit >= target) || S2.picard_iter >= ip2.maxiter_nonlinear;
      if (done) {
        S2.picard_converged = S2.picard_iter < ip2.maxiter_nonlinear ? 1 : 0;
        S2.picard_active = 0;
        atomicSub(&v.cnt->picard_active, 1);
      }
    };
    if (meanu) tile_finish<2, false>(v, t, R.inst, part, fin);
    else tile_finish<2, true>(v, t, R.inst, part, fin);
  }
}

// ---------------------------------------------------------------------
// Mixed precision: FP32 copy of the symmetric matrix for the Krylov
// iteration; the every-ncheck true residual r = b - A x stays FP64, so the
// iteration is a reliable-update PCG that converges to the FP64 solution.
// ---------------------------------------------------------------------
// FP32 copy of the symmetric matrix with the row-sum compensated FP64
// diagonal block (make_a32_row).
__global__ void __launch_bounds__(kTile) k_make_a32(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (!tile_mine(v, R, threadIdx.x)) continue;
    const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
    make_a32_row(v, col, k, (size_t)n);
  }
}

// Factors of the SIA column preconditioner for the linear solve ahead:
// one thread per (column, component) of the instances that use it and are
// solving (sia_factor_column).
__global__ void __launch_bounds__(256) k_sia_factor(DevView v) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2L * v.ncols) return;
  const int col = (int)(t >> 1), h = (int)(t & 1);
  const int inst = v.col_inst[col];
  if (v.inst[inst].precond != 2 || !v.st[inst].pcg_active) return;
  sia_factor_column(v, col, h);
}

// Post-solve diagnostics (glissade_velo_higher.F90:3847-3872) at the
// current velocity: the element stresses of compute_internal_stress into
// out[6][nelem] (a singular Jacobian marks the instance, as assembly pass 1
// does) and the basal frictional heat flux of
// compute_basal_friction_heatflx into bf (per active cell for the
// finite-element method, per column for the local one).
__global__ void __launch_bounds__(256) k_internal_stress(DevView v, double* out) {
  const size_t ne = (size_t)v.nelem;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < v.nelem; e += gridDim.x * blockDim.x) {
    double tau[6];
    if (!stress_element(v, c_T, e, tau)) {
      atomicExch(&v.st[v.cell_inst[e / (v.nz - 1)]].status, BP_ERR_SINGULAR_JAC);
      for (int q = 0; q < 6; ++q) tau[q] = 0.0;
    }
    for (int q = 0; q < 6; ++q) out[(size_t)q * ne + e] = tau[q];
  }
}

__global__ void __launch_bounds__(256) k_bfric(DevView v, int which, double* bf) {
  const int n = which == 0 ? v.ncells : v.ncols;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    bf[i] = which == 0 ? bfric_cell(v, c_T, i) : bfric_vertex(v, i);
}

// Plain y = A x for bp_matvec.
__global__ void __launch_bounds__(kTile) k_matvec_plain(DevView v, const double2* x, double2* y) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const int n = R.n0 + threadIdx.x;
    if (!tile_mine(v, R, threadIdx.x)) continue;
    const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
    y[n] = v.sym ? matvec_row_sym(v, v.A, col, k, n, SrcX{x}) : matvec_row(v, v.A, col, k, n, SrcX{x});
  }
}

// y = A x for the autotuner and the kernel sweep: one storage variant and
// one occupancy target (MINB = minimum resident CTAs per SM, 0 = free).
template <int STORE, int MINB>
__global__ void __launch_bounds__(kTile, MINB) k_tune_mv(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const int n = R.n0 + threadIdx.x;
    if (!tile_mine(v, R, threadIdx.x)) continue;
    const int col = tile_col(v, R, threadIdx.x), k = tile_k(v, threadIdx.x);
    v.Az[n] = mv_row<STORE>(v, col, k, n, v.x);
  }
}

// Diagonal preconditioner for matrix-level entry points.
__global__ void __launch_bounds__(kTile) k_dinv(DevView v, int precond) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const int n = R.n0 + threadIdx.x;
    if (!tile_mine(v, R, threadIdx.x)) continue;
    const size_t np = (size_t)v.npad;
    double2 di = make_double2(1.0, 1.0);
    (void)np;
    if (precond == 1) {
      const double du = diag_u(v, n), dv = diag_v(v, n);
      di.x = du != 0.0 ? 1.0 / du : 0.0;
      di.y = dv != 0.0 ? 1.0 / dv : 0.0;
    }
    v.Dinv[n] = di;
  }
}

// (b,b) for matrix-level entry points.
__global__ void __launch_bounds__(kTile) k_bb(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const int n = R.n0 + threadIdx.x;
    double part[1] = {0.0};
    if (tile_mine(v, R, threadIdx.x)) {
      const double2 b = v.b[n];
      part[0] = b.x * b.x + b.y * b.y;
    }
    tile_finish<1, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      v.st[inst].bb = s[0];
      v.st[inst].L2_rhs = sqrt(s[0]);
    });
  }
}

// ---------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------
static inline int tile_grid(const DevView& v) {
  int g = v.ntiles > 0 ? v.ntiles : 1;
  if (v.grid_cap > 0 && g > v.grid_cap) g = v.grid_cap;
  return g;
}

cudaError_t upload_ref_tables() {
  RefTables t;
  fill_ref_tables(&t);
  return cudaMemcpyToSymbol(c_T, &t, sizeof(t));
}

void launch_picard_begin(const DevView& v, cudaStream_t s) { k_picard_begin<<<1, 256, 0, s>>>(v); }
void launch_save_usav(const DevView& v, cudaStream_t s) { k_save_usav<<<tile_grid(v), v.tile_threads, 0, s>>>(v); }
void launch_slide_beta(const DevView& v, cudaStream_t s) {
  if (v.ncols > 0) k_slide_beta<<<(v.ncols + kTile - 1) / kTile, kTile, 0, s>>>(v);
  if (v.ncells > 0) k_cell_beta<<<(v.ncells + kTile - 1) / kTile, kTile, 0, s>>>(v);
}
void launch_asm_qp(const DevView& v, cudaStream_t s) {
  if (v.solve2d) {
    if (v.ncells > 0) {
      const long threads = (long)v.ncells * 4;
      if (v.l1l2 || v.diva) k_asm2_qp<true><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(v);
      else k_asm2_qp<false><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(v);
    }
  } else if (v.nelem > 0) {
    const long threads = (long)v.nelem * 8;
    k_asm_qp<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(v);
  }
}
void launch_asm_rows(const DevView& v, cudaStream_t s) {
  dim3 g(tile_grid(v), 4);
  if (v.solve2d) {
    k_asm_rows<ASM_2D><<<g, v.tile_threads, 0, s>>>(v);
  } else if (v.Ke) {
    if (v.nelem > 0) k_asm_elem<<<(unsigned)(((long)v.nelem * 8 + 255) / 256), 256, 0, s>>>(v);
    k_asm_rows<ASM_GATHER><<<g, v.tile_threads, 0, s>>>(v);
  } else {
    k_asm_rows<ASM_ROWS><<<g, v.tile_threads, 0, s>>>(v);
  }
}
void launch_rhs(const DevView& v, cudaStream_t s) { k_rhs<<<tile_grid(v), v.tile_threads, 0, s>>>(v); }
void launch_diva_beta(const DevView& v, cudaStream_t s) {
  if (v.ncells > 0) k_diva_cells<<<(unsigned)((v.ncells + 255) / 256), 256, 0, s>>>(v);
  if (v.ncols > 0) k_diva_beta<<<(unsigned)((v.ncols + 255) / 256), 256, 0, s>>>(v);
  if (v.ncells > 0) k_diva_cell_beta<<<(unsigned)((v.ncells + 255) / 256), 256, 0, s>>>(v);
}
void launch_diva_velocity(const DevView& v, cudaStream_t s) {
  if (v.ncols > 0) k_diva_velocity<<<(unsigned)((v.ncols + 255) / 256), 256, 0, s>>>(v);
}
void launch_l1l2_velocity(const DevView& v, cudaStream_t s) {
  if (v.ncells > 0) k_l1l2_cells<<<(unsigned)((v.ncells + 255) / 256), 256, 0, s>>>(v);
  if (v.ncols > 0) k_l1l2_columns<<<(unsigned)((v.ncols + 255) / 256), 256, 0, s>>>(v);
}
void launch_assemble(const DevView& v, cudaStream_t s) {
  launch_asm_qp(v, s);
  launch_asm_rows(v, s);
  launch_rhs(v, s);
}
// PCG kernels are launched as programmatic dependents of their stream
// predecessor (BP_PDL=0 turns this off, and so does set_pdl(false), e.g.
// while a graph that cannot hold programmatic edges is captured), and with
// the problem's L2 access-policy window when it has one.
static const bool g_pdl_env = [] {
  const char* e = std::getenv("BP_PDL");
  return !(e && e[0] == '0');
}();
static thread_local bool g_pdl_on = true;
void set_pdl(bool on) { g_pdl_on = on; }

static void launch_pcg(void (*kernel)(DevView), int g, cudaStream_t s, const DevView& v, int block = 0) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g);
  cfg.blockDim = dim3(block > 0 ? block : v.tile_threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  unsigned na = 0;
  if (g_pdl_env && g_pdl_on) {
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  if (v.l2_bytes > 0) {
    at[na].id = cudaLaunchAttributeAccessPolicyWindow;
    at[na].val.accessPolicyWindow.base_ptr = const_cast<void*>(v.l2_base);
    at[na].val.accessPolicyWindow.num_bytes = v.l2_bytes;
    at[na].val.accessPolicyWindow.hitRatio = v.l2_hit;
    at[na].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    at[na].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    ++na;
  }
  cfg.attrs = at;
  cfg.numAttrs = na;
  cudaLaunchKernelEx(&cfg, kernel, v);
}

using TileKernel = void (*)(DevView);

template <int STORE, int MINB>
static void launch_resid_store(int mode, const DevView& v, cudaStream_t s, int g) {
  switch (mode) {
    case MV_INIT: launch_pcg(k_resid<MV_INIT, STORE, MINB>, g, s, v); break;
    case MV_CHECK: launch_pcg(k_resid<MV_CHECK, STORE, MINB>, g, s, v); break;
    default: launch_pcg(k_resid<MV_REFINE, STORE, MINB>, g, s, v); break;
  }
}
template <int STORE, int MINB>
static TileKernel krylov_kernel(int mode) {
  switch (mode) {
    case MV_STD_A: return k_std_mv<STORE, MINB>;
    case MV_CG_FIRST: return k_cg_mv<true, STORE, MINB>;
    default: return k_cg_mv<false, STORE, MINB>;
  }
}
template <int STORE>
static TileKernel krylov_kernel_st(int mode, int minb) {
  if (minb == 8) return krylov_kernel<STORE, 8>(mode);
  if (minb == 6) return krylov_kernel<STORE, 6>(mode);
  if (minb == 4) return krylov_kernel<STORE, 4>(mode);
  return krylov_kernel<STORE, 0>(mode);
}
static TileKernel krylov_kernel_for(const DevView& v, int mode, int minb) {
  if (!v.sym) return krylov_kernel_st<ST_FULL>(mode, minb);
  if (v.A32) return krylov_kernel_st<ST_SYM32>(mode, minb);
  return krylov_kernel_st<ST_SYM>(mode, minb);
}
static inline bool is_krylov(int mode) {
  return mode == MV_STD_A || mode == MV_CG_FIRST || mode == MV_CG1;
}
template <int STORE>
static void launch_resid_minb(int mode, const DevView& v, cudaStream_t s, int g) {
  if (v.minb == 4) launch_resid_store<STORE, 4>(mode, v, s, g);
  else launch_resid_store<STORE, 0>(mode, v, s, g);
}
void launch_mv(int mode, const DevView& v, cudaStream_t s) {
  if (is_krylov(mode)) {
    int g = v.ntiles > 0 ? v.ntiles : 1;
    if (v.grid_k > 0 && g > v.grid_k) g = v.grid_k;
    launch_pcg(krylov_kernel_for(v, mode, v.minb_k), g, s, v);
    return;
  }
  const int g = tile_grid(v);
  if (!v.sym) launch_resid_minb<ST_FULL>(mode, v, s, g);
  else if (v.A32) launch_resid_minb<ST_SYM32>(mode, v, s, g);
  else launch_resid_minb<ST_SYM>(mode, v, s, g);
}
int krylov_resident_ctas(const DevView& v, int mode, int minb) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, krylov_kernel_for(v, mode, minb), v.tile_threads, 0) !=
      cudaSuccess)
    return 0;
  return n;
}
void launch_std_update(bool check, const DevView& v, cudaStream_t s) {
  launch_pcg(check ? k_std_update<true> : k_std_update<false>, tile_grid(v), s, v);
}
void launch_std_dir(const DevView& v, cudaStream_t s) { launch_pcg(k_std_dir, tile_grid(v), s, v); }
void launch_cg_first_update(const DevView& v, cudaStream_t s) {
  launch_pcg(k_cg_first_update, tile_grid(v), s, v);
}
void launch_cg_update(bool check, const DevView& v, cudaStream_t s) {
  launch_pcg(check ? k_cg_update<true> : k_cg_update<false>, tile_grid(v), s, v);
}
void launch_picard_check(const DevView& v, cudaStream_t s) {
  k_picard_check<<<tile_grid(v), v.tile_threads, 0, s>>>(v);
}

// Conditions of the device-resident loops (CUDA-graph WHILE nodes).  One
// thread: count this pass in *iter (reset to 0 by `reset`) and keep
// looping while some instance is active (counter *active > 0) and fewer
// than `cap` passes ran, so every loop ends after at most `cap` passes.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const int* active, int* iter, int cap, int reset) {
  const int it = reset ? (*iter = 0) : ++*iter;
  cudaGraphSetConditional(h, (*active > 0 && it < cap) ? 1u : 0u);
}
void launch_loop_cond(cudaGraphConditionalHandle h, const DevView& v, bool picard, int* iter, int cap, bool reset,
                      cudaStream_t s) {
  const int* active = picard ? &v.cnt->picard_active : &v.cnt->pcg_active;
  k_loop_cond<<<1, 1, 0, s>>>(h, active, iter, cap, reset ? 1 : 0);
}
void launch_make_a32(const DevView& v, cudaStream_t s) { k_make_a32<<<tile_grid(v), v.tile_threads, 0, s>>>(v); }
void launch_sia_factor(const DevView& v, cudaStream_t s) {
  if (v.sia_f && v.ncols > 0) k_sia_factor<<<(unsigned)((2L * v.ncols + 255) / 256), 256, 0, s>>>(v);
}
void launch_matvec_plain(const DevView& v, const double2* x, double2* y, cudaStream_t s) {
  k_matvec_plain<<<tile_grid(v), v.tile_threads, 0, s>>>(v, x, y);
}
void launch_dinv(const DevView& v, int precond, cudaStream_t s) {
  k_dinv<<<tile_grid(v), v.tile_threads, 0, s>>>(v, precond);
}
void launch_bb(const DevView& v, cudaStream_t s) { k_bb<<<tile_grid(v), v.tile_threads, 0, s>>>(v); }
// The 3-D velocity of a shallow-shelf solve (its 2-D solution on every
// level, :3745-3750) for the post-solve diagnostics.
__global__ void __launch_bounds__(256) k_levels_from_2d(DevView v, double2* x3, int L) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (long)v.ncols * L) x3[t] = v.x[v.col_node[t / L]];
}

// The bed-face corner betas from the columns' beta_internal (0 where a
// corner has no column) for every cell.
__global__ void __launch_bounds__(256) k_corner_beta(DevView v) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= v.ncells) return;
  for (int q = 0; q < 4; ++q) {
    const int col = v.cell_cols[(size_t)q * v.ncells + cell];
    v.cell_beta[(size_t)q * v.ncells + cell] = col >= 0 ? v.col_beta[col] : 0.0;
  }
}

void launch_levels_from_2d(const DevView& v, double2* x3, int L, cudaStream_t s) {
  const long n = (long)v.ncols * L;
  if (n > 0) k_levels_from_2d<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v, x3, L);
}
void launch_corner_beta(const DevView& v, cudaStream_t s) {
  if (v.ncells > 0) k_corner_beta<<<(unsigned)((v.ncells + 255) / 256), 256, 0, s>>>(v);
}

void launch_diagnostics(const DevView& v, int which_bfric, double* tau, double* bf, cudaStream_t s) {
  if (tau && v.nelem > 0) k_internal_stress<<<(v.nelem + 255) / 256, 256, 0, s>>>(v, tau);
  const int n = which_bfric == 0 ? v.ncells : v.ncols;
  if (bf && n > 0) k_bfric<<<(n + 255) / 256, 256, 0, s>>>(v, which_bfric, bf);
}
int launch_tune_mv(int store, int minb, int grid, const DevView& v, cudaStream_t s) {
  const int g = grid > 0 ? grid : tile_grid(v);
#define TUNE(ST, MB) k_tune_mv<ST, MB><<<g, v.tile_threads, 0, s>>>(v)
  if (store == ST_FULL && !v.sym) {
    if (minb == 8) TUNE(ST_FULL, 8); else if (minb == 6) TUNE(ST_FULL, 6);
    else if (minb == 4) TUNE(ST_FULL, 4); else TUNE(ST_FULL, 0);
  } else if (store == ST_SYM && v.sym) {
    if (minb == 8) TUNE(ST_SYM, 8); else if (minb == 6) TUNE(ST_SYM, 6);
    else if (minb == 4) TUNE(ST_SYM, 4); else TUNE(ST_SYM, 0);
  } else if (store == ST_SYM32 && v.sym && v.A32) {
    if (minb == 8) TUNE(ST_SYM32, 8); else if (minb == 6) TUNE(ST_SYM32, 6);
    else if (minb == 4) TUNE(ST_SYM32, 4); else TUNE(ST_SYM32, 0);
  } else {
    return -1;
  }
#undef TUNE
  return 0;
}

}  // namespace bp
