// bp_kernels.cu -- sm_100a kernels of the Blatter-Pattyn solve.
//
// All node kernels walk tiles of kTile consecutive nodes (one tile per CTA
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
  int inst, n0, nend;
};

__device__ __forceinline__ TileRange tile_range(const DevView& v, int t) {
  TileRange r;
  r.inst = v.tile_inst[t];
  r.n0 = v.tile_start[t];
  r.nend = min(r.n0 + kTile, v.inst[r.inst].node_end);
  return r;
}

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
    ++mine;
  }
  atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    v.cnt->pcg_active = cnt;
    v.cnt->refine_active = cnt;
  }
}

__global__ void __launch_bounds__(kTile) k_save_usav(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].picard_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (n < R.nend) v.usav[n] = v.x[n];
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

// ---------------------------------------------------------------------
// Assembly pass 2 + basal BC + Dirichlet BC: thread = (block B, node).
// ---------------------------------------------------------------------
template <int B>
__device__ __forceinline__ bool asm_row(const DevView& v, int n) {
  const int col = n / v.nz, k = n - col * v.nz;
  double acc[27];
  row_assemble<B>(v, c_T, col, k, acc);
  row_basal<B>(v, c_T, col, k, acc);
  const double adj = row_dirichlet<B>(v, col, k, acc);
  bool nz = false;
  double* Ad = reinterpret_cast<double*>(v.A);
  const size_t np = (size_t)v.npad;
  const int h = B >> 1, comp = B & 1;
#pragma unroll
  for (int m = 0; m < 27; ++m) {
    nz |= (acc[m] != 0.0);
    Ad[(((size_t)(h * 27 + m)) * np + n) * 2 + comp] = acc[m];
  }
  v.badj[(size_t)B * np + n] = adj;
  return nz;
}

__global__ void __launch_bounds__(kTile) k_asm_rows(DevView v) {
  const int B = blockIdx.y;
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].picard_active) continue;
    const int n = R.n0 + threadIdx.x;
    int nzl = 0;
    if (n < R.nend) {
      switch (B) {
        case 0: nzl = asm_row<0>(v, n); break;
        case 1: nzl = asm_row<1>(v, n); break;
        case 2: nzl = asm_row<2>(v, n); break;
        default: nzl = asm_row<3>(v, n); break;
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
    if (n < R.nend) {
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
        const double du = v.A[13 * np + n].x, dv = v.A[(27 + 13) * np + n].y;
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
      if (S.status == BP_ERR_SINGULAR_JAC) {
        fail(v, S, BP_ERR_SINGULAR_JAC);
      } else if (!S.nonzero) {
        S.status = BP_ZERO_MATRIX;
        S.zero_x = 1;
        fail(v, S, BP_ZERO_MATRIX);
      }
    });
  }
}

// ---------------------------------------------------------------------
// Fused matvec kernels.  Source vectors are formed on the fly at the
// node and its neighbours (z = D^-1 r, d = z + beta d_old) so no separate
// preconditioner or direction-update pass is needed.
// ---------------------------------------------------------------------
struct SrcX {
  const double2* x;
  __device__ double2 operator()(size_t m) const { return x[m]; }
};
struct SrcZ {  // z = D^-1 r
  const double2 *r, *di;
  __device__ double2 operator()(size_t m) const {
    const double2 a = r[m], b = di[m];
    return make_double2(a.x * b.x, a.y * b.y);
  }
};
struct SrcD {  // d = z + beta d_old
  const double2 *r, *di, *dold;
  double beta;
  bool first;
  __device__ double2 operator()(size_t m) const {
    const double2 a = r[m], b = di[m];
    double2 z = make_double2(a.x * b.x, a.y * b.y);
    if (!first) {
      const double2 o = dold[m];
      z.x = z.x + beta * o.x;
      z.y = z.y + beta * o.y;
    }
    return z;
  }
};

template <int MODE>
__global__ void __launch_bounds__(kTile) k_mv(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const InstParams& ip = v.inst[R.inst];
    const int n = R.n0 + threadIdx.x;
    const int it = S.pcg_iter;
    double part[2] = {0.0, 0.0};
    if (n < R.nend) {
      const int col = n / v.nz, k = n - col * v.nz;
      if (MODE == MV_INIT || MODE == MV_CHECK) {
        const double2 y = matvec_row(v, v.A, col, k, n, SrcX{v.x});
        const double2 b = v.b[n], di = v.Dinv[n];
        const double ru = b.x - y.x, rv = b.y - y.y;
        v.r[n] = make_double2(ru, rv);
        part[0] = ru * (ru * di.x) + rv * (rv * di.y);  // (r, z)
        part[1] = ru * ru + rv * rv;                    // (r, r)
      } else if (MODE == MV_STD_A) {
        double2* dold = (it & 1) ? v.d0 : v.d1;
        double2* dnew = (it & 1) ? v.d1 : v.d0;
        const SrcD src{v.r, v.Dinv, dold, S.beta, it == 1};
        const double2 y = matvec_row(v, v.A, col, k, n, src);
        const double2 d = src((size_t)n);
        dnew[n] = d;
        v.q[n] = y;
        part[0] = d.x * y.x + d.y * y.y;
      } else if (MODE == MV_CG_FIRST) {
        const SrcZ src{v.r, v.Dinv};
        const double2 y = matvec_row(v, v.A, col, k, n, src);
        const double2 z = src((size_t)n), r = v.r[n];
        v.d0[n] = z;
        v.q[n] = y;
        part[0] = r.x * z.x + r.y * z.y;
        part[1] = z.x * y.x + z.y * y.y;
      } else if (MODE == MV_CG1) {
        const SrcZ src{v.r, v.Dinv};
        const double2 y = matvec_row(v, v.A, col, k, n, src);
        const double2 z = src((size_t)n), r = v.r[n];
        v.Az[n] = y;
        part[0] = r.x * z.x + r.y * z.y;
        part[1] = y.x * z.x + y.y * z.y;
      }
    }
    tile_finish<2, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      InstState& S2 = v.st[inst];
      const InstParams& ip2 = v.inst[inst];
      if (MODE == MV_INIT) {
        S2.L2_norm = sqrt(s[1]);
        S2.L2_rel = S2.L2_rhs > 0.0 ? S2.L2_norm / S2.L2_rhs : 0.0;
        if (ip2.variant != 3) {  // standard PCG: eta1 of iteration 1
          if (is_nan(s[0])) { fail(v, S2, BP_ERR_NAN); return; }
          S2.beta = s[0] / S2.rz;
          S2.rz = s[0];
        }
      } else if (MODE == MV_STD_A) {
        const double alpha = S2.rz / s[0];
        if (is_nan(alpha)) { fail(v, S2, BP_ERR_NAN); return; }
        S2.alpha = alpha;
      } else if (MODE == MV_CG_FIRST) {
        S2.rz_old = s[0];
        S2.sigma = s[1];
        const double alpha = s[0] / s[1];
        if (is_nan(alpha)) { fail(v, S2, BP_ERR_NAN); return; }
        S2.alpha = alpha;
      } else if (MODE == MV_CG1) {
        S2.pcg_iter += 1;
        if (S2.pcg_iter > ip2.pcg_maxiters) {
          S2.pcg_iter = ip2.pcg_maxiters;
          pcg_stop(v, S2, false);
          return;
        }
        const double rho = s[0], delta = s[1];
        const double beta = rho / S2.rz_old;
        const double sigma = delta - beta * rho / S2.alpha;
        const double alpha = rho / sigma;
        S2.rz_old = rho;
        S2.beta = beta;
        S2.sigma = sigma;
        if (is_nan(alpha)) { fail(v, S2, BP_ERR_NAN); return; }
        S2.alpha = alpha;
      } else if (MODE == MV_CHECK) {
        S2.err = sqrt(s[1]) / S2.L2_rhs;
        if (S2.err < ip2.pcg_tol) { pcg_stop(v, S2, true); return; }
        if (S2.pcg_iter >= ip2.pcg_maxiters) { pcg_stop(v, S2, false); return; }
        if (ip2.variant != 3) {
          if (is_nan(s[0])) { fail(v, S2, BP_ERR_NAN); return; }
          S2.beta = s[0] / S2.rz;
          S2.rz = s[0];
          S2.pcg_iter += 1;
        }
      }
    });
  }
}

// Standard PCG update: x += alpha d; r -= alpha q; (r, D^-1 r).
template <bool CHECK>
__global__ void __launch_bounds__(kTile) k_std_update(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    const int it = S.pcg_iter;
    const double alpha = S.alpha;
    double part[1] = {0.0};
    if (n < R.nend) {
      const double2 d = ((it & 1) ? v.d1 : v.d0)[n];
      double2 x = v.x[n];
      x.x = x.x + alpha * d.x;
      x.y = x.y + alpha * d.y;
      v.x[n] = x;
      if (!CHECK) {
        const double2 q = v.q[n], di = v.Dinv[n];
        double2 r = v.r[n];
        r.x = r.x - alpha * q.x;
        r.y = r.y - alpha * q.y;
        v.r[n] = r;
        part[0] = r.x * (r.x * di.x) + r.y * (r.y * di.y);
      }
    }
    if (!CHECK) {
      tile_finish<1, false>(v, t, R.inst, part, [&](int inst, const double* s) {
        InstState& S2 = v.st[inst];
        if (S2.pcg_iter >= v.inst[inst].pcg_maxiters) { pcg_stop(v, S2, false); return; }
        if (is_nan(s[0])) { fail(v, S2, BP_ERR_NAN); return; }
        S2.beta = s[0] / S2.rz;
        S2.rz = s[0];
        S2.pcg_iter += 1;
      });
    }
  }
}

// Chronopoulos-Gear first-pass update: x += alpha d; r -= alpha q.
__global__ void __launch_bounds__(kTile) k_cg_first_update(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const double alpha = S.alpha;
    const double2 d = v.d0[n], q = v.q[n];
    double2 x = v.x[n], r = v.r[n];
    x.x = x.x + alpha * d.x; x.y = x.y + alpha * d.y;
    r.x = r.x - alpha * q.x; r.y = r.y - alpha * q.y;
    v.x[n] = x;
    v.r[n] = r;
  }
}

// Chronopoulos-Gear loop update: d = z + beta d; q = Az + beta q;
// x += alpha d; r -= alpha q (glissade_velo_higher_pcg.F90:1519-1534).
template <bool CHECK>
__global__ void __launch_bounds__(kTile) k_cg_update(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const double alpha = S.alpha, beta = S.beta;
    const double2 r = v.r[n], di = v.Dinv[n], az = v.Az[n];
    double2 d = v.d0[n], q = v.q[n], x = v.x[n];
    const double zu = r.x * di.x, zv = r.y * di.y;
    d.x = zu + beta * d.x; d.y = zv + beta * d.y;
    q.x = az.x + beta * q.x; q.y = az.y + beta * q.y;
    x.x = x.x + alpha * d.x; x.y = x.y + alpha * d.y;
    v.d0[n] = d;
    v.q[n] = q;
    v.x[n] = x;
    if (!CHECK) v.r[n] = make_double2(r.x - alpha * q.x, r.y - alpha * q.y);
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
    if (S.zero_x) {
      if (n < R.nend) v.x[n] = make_double2(0.0, 0.0);
      continue;
    }
    if (!S.picard_active) continue;
    const bool meanu = ip.which_resid == 2;
    const bool nobed = ip.which_resid == 1 || meanu;
    double part[2] = {0.0, 0.0};
    if (n < R.nend) {
      const int k = n % v.nz;
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
// Mixed precision: FP32 equilibrated matrix, FP32 inner CG with FP64
// reductions, FP64 iterative refinement.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) k_scale(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const size_t np = (size_t)v.npad;
    const double du = v.A[13 * np + n].x, dv = v.A[(27 + 13) * np + n].y;
    v.scale[n] = make_double2(du > 0.0 ? 1.0 / sqrt(du) : 0.0, dv > 0.0 ? 1.0 / sqrt(dv) : 0.0);
  }
}

__global__ void __launch_bounds__(kTile) k_make_a32(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const int nz = v.nz, nc = v.ncols;
    const int col = n / nz, k = n - col * nz;
    const size_t np = (size_t)v.npad;
    const double2 sn = v.scale[n];
#pragma unroll
    for (int kA = -1; kA <= 1; ++kA)
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        const int m = (kA + 1) * 9 + q;
        const int cn = v.col_nbr[q * nc + col];
        const int kn = k + kA;
        double2 sm = make_double2(0.0, 0.0);
        if (cn >= 0 && kn >= 0 && kn < nz) sm = v.scale[(size_t)cn * nz + kn];
        const double2 au = v.A[(size_t)m * np + n], av = v.A[(size_t)(27 + m) * np + n];
        v.A32[(size_t)m * np + n] =
            make_float2((float)(sn.x * au.x * sm.x), (float)(sn.x * au.y * sm.y));
        v.A32[(size_t)(27 + m) * np + n] =
            make_float2((float)(sn.y * av.x * sm.x), (float)(sn.y * av.y * sm.y));
      }
  }
}

// Outer residual r = b - A x (FP64); start of an inner solve.
__global__ void __launch_bounds__(kTile) k_refine_resid(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    InstState& S = v.st[R.inst];
    if (!S.refine_active) continue;
    const int n = R.n0 + threadIdx.x;
    double part[2] = {0.0, 0.0};
    if (n < R.nend) {
      const int col = n / v.nz, k = n - col * v.nz;
      const double2 y = matvec_row(v, v.A, col, k, n, SrcX{v.x});
      const double2 b = v.b[n], s = v.scale[n];
      const double ru = b.x - y.x, rv = b.y - y.y;
      const float su = (float)(s.x * ru), sv = (float)(s.y * rv);
      v.r32[n] = make_float2(su, sv);
      v.y32[n] = make_float2(0.f, 0.f);
      part[0] = ru * ru + rv * rv;
      part[1] = (double)su * su + (double)sv * sv;
    }
    tile_finish<2, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      InstState& S2 = v.st[inst];
      const InstParams& ip2 = v.inst[inst];
      S2.err = S2.L2_rhs > 0.0 ? sqrt(s[0]) / S2.L2_rhs : 0.0;
      if (S2.refine_steps == 0) {
        S2.L2_norm = sqrt(s[0]);
        S2.L2_rel = S2.err;
      }
      const bool conv = !(S2.err >= ip2.pcg_tol);
      if (conv || S2.refine_steps >= 20 || S2.pcg_iters_last >= ip2.pcg_maxiters || is_nan(s[0])) {
        S2.refine_active = 0;
        S2.pcg_active = 0;
        S2.pcg_converged = conv ? 1 : 0;
        S2.refine_steps_total += S2.refine_steps;
        S2.pcg_iters_total += S2.pcg_iters_last;
        atomicSub(&v.cnt->refine_active, 1);
        if (is_nan(s[0])) fail(v, S2, BP_ERR_NAN);
        return;
      }
      S2.refine_steps += 1;
      S2.in_rr0 = s[1];
      S2.rz = s[1];
      S2.beta = 0.0;
      S2.inner_iter = 1;
      S2.pcg_active = 1;
      atomicAdd(&v.cnt->pcg_active, 1);
    });
  }
}

struct SrcP32 {  // p = r + beta p_old, FP32 storage
  const float2 *r, *pold;
  float beta;
  bool first;
  __device__ float2 operator()(size_t m) const {
    const float2 a = r[m];
    if (first) return a;
    const float2 o = pold[m];
    return make_float2(a.x + beta * o.x, a.y + beta * o.y);
  }
};

template <typename Src>
__device__ __forceinline__ float2 matvec_row32(const DevView& v, int col, int k, size_t n,
                                               const Src& src) {
  const int nz = v.nz, nc = v.ncols;
  const size_t np = (size_t)v.npad;
  int cn[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) cn[q] = v.col_nbr[q * nc + col];
  float yu = 0.f, yv = 0.f;
#pragma unroll
  for (int kA = -1; kA <= 1; ++kA) {
    const int kn = k + kA;
    if (kn < 0 || kn >= nz) continue;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      if (cn[q] < 0) continue;
      const int m = (kA + 1) * 9 + q;
      const float2 au = __ldcs(v.A32 + (size_t)m * np + n);
      const float2 av = __ldcs(v.A32 + (size_t)(27 + m) * np + n);
      const float2 s = src((size_t)cn[q] * nz + kn);
      yu = fmaf(au.x, s.x, fmaf(au.y, s.y, yu));
      yv = fmaf(av.x, s.x, fmaf(av.y, s.y, yv));
    }
  }
  return make_float2(yu, yv);
}

// Inner CG, part A: p = r + beta p_old; q = A32 p; (p, q).
__global__ void __launch_bounds__(kTile) k_inner_a(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    const int it = S.inner_iter;
    double part[1] = {0.0};
    if (n < R.nend) {
      const int col = n / v.nz, k = n - col * v.nz;
      float2* pold = (it & 1) ? v.p32a : v.p32b;
      float2* pnew = (it & 1) ? v.p32b : v.p32a;
      const SrcP32 src{v.r32, pold, (float)S.beta, it == 1};
      const float2 y = matvec_row32(v, col, k, n, src);
      const float2 p = src((size_t)n);
      pnew[n] = p;
      v.q32[n] = y;
      part[0] = (double)p.x * y.x + (double)p.y * y.y;
    }
    tile_finish<1, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      InstState& S2 = v.st[inst];
      const double alpha = S2.rz / s[0];
      if (is_nan(alpha) || !(s[0] > 0.0)) {  // breakdown: end this inner solve
        S2.alpha = 0.0;
        S2.pcg_active = 0;
        atomicSub(&v.cnt->pcg_active, 1);
        return;
      }
      S2.alpha = alpha;
    });
  }
}

// Inner CG, part B: y += alpha p; r -= alpha q; (r, r); inner stop test.
__global__ void __launch_bounds__(kTile) k_inner_b(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    InstState& S = v.st[R.inst];
    if (!S.pcg_active) continue;
    const int n = R.n0 + threadIdx.x;
    const int it = S.inner_iter;
    const float alpha = (float)S.alpha;
    double part[1] = {0.0};
    if (n < R.nend) {
      const float2 p = ((it & 1) ? v.p32b : v.p32a)[n];
      const float2 q = v.q32[n];
      float2 y = v.y32[n], r = v.r32[n];
      y.x = fmaf(alpha, p.x, y.x); y.y = fmaf(alpha, p.y, y.y);
      r.x = fmaf(-alpha, q.x, r.x); r.y = fmaf(-alpha, q.y, r.y);
      v.y32[n] = y;
      v.r32[n] = r;
      part[0] = (double)r.x * r.x + (double)r.y * r.y;
    }
    tile_finish<1, false>(v, t, R.inst, part, [&](int inst, const double* s) {
      InstState& S2 = v.st[inst];
      const InstParams& ip2 = v.inst[inst];
      S2.pcg_iters_last += 1;
      const double tol = ip2.inner_tol;
      if (!(s[0] > tol * tol * S2.in_rr0) || S2.pcg_iters_last >= ip2.pcg_maxiters) {
        S2.pcg_active = 0;
        atomicSub(&v.cnt->pcg_active, 1);
        return;
      }
      S2.beta = s[0] / S2.rz;
      S2.rz = s[0];
      S2.inner_iter += 1;
    });
  }
}

// x += S y after an inner solve.
__global__ void __launch_bounds__(kTile) k_refine_update(DevView v) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    if (!v.st[R.inst].refine_active) continue;
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const float2 y = v.y32[n];
    const double2 s = v.scale[n];
    double2 x = v.x[n];
    x.x += s.x * (double)y.x;
    x.y += s.y * (double)y.y;
    v.x[n] = x;
  }
}

// Plain y = A x for bp_matvec.
__global__ void __launch_bounds__(kTile) k_matvec_plain(DevView v, const double2* x, double2* y) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const int col = n / v.nz, k = n - col * v.nz;
    y[n] = matvec_row(v, v.A, col, k, n, SrcX{x});
  }
}

// Diagonal preconditioner for matrix-level entry points.
__global__ void __launch_bounds__(kTile) k_dinv(DevView v, int precond) {
  for (int t = blockIdx.x; t < v.ntiles; t += gridDim.x) {
    const TileRange R = tile_range(v, t);
    const int n = R.n0 + threadIdx.x;
    if (n >= R.nend) continue;
    const size_t np = (size_t)v.npad;
    double2 di = make_double2(1.0, 1.0);
    if (precond == 1) {
      const double du = v.A[13 * np + n].x, dv = v.A[(27 + 13) * np + n].y;
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
    if (n < R.nend) {
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
static int g_grid_cap = 0;

void set_grid_cap(int cap) { g_grid_cap = cap; }

static inline int tile_grid(const DevView& v) {
  int g = v.ntiles > 0 ? v.ntiles : 1;
  if (g_grid_cap > 0 && g > g_grid_cap) g = g_grid_cap;
  return g;
}

cudaError_t upload_ref_tables() {
  RefTables t;
  fill_ref_tables(&t);
  return cudaMemcpyToSymbol(c_T, &t, sizeof(t));
}

void launch_picard_begin(const DevView& v, cudaStream_t s) { k_picard_begin<<<1, 256, 0, s>>>(v); }
void launch_save_usav(const DevView& v, cudaStream_t s) { k_save_usav<<<tile_grid(v), kTile, 0, s>>>(v); }
void launch_asm_qp(const DevView& v, cudaStream_t s) {
  if (v.nelem > 0) {
    const long threads = (long)v.nelem * 8;
    k_asm_qp<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(v);
  }
}
void launch_asm_rows(const DevView& v, cudaStream_t s) {
  dim3 g(tile_grid(v), 4);
  k_asm_rows<<<g, kTile, 0, s>>>(v);
}
void launch_rhs(const DevView& v, cudaStream_t s) { k_rhs<<<tile_grid(v), kTile, 0, s>>>(v); }
void launch_assemble(const DevView& v, cudaStream_t s) {
  launch_asm_qp(v, s);
  launch_asm_rows(v, s);
  launch_rhs(v, s);
}
void launch_mv(int mode, const DevView& v, cudaStream_t s) {
  const int g = tile_grid(v);
  switch (mode) {
    case MV_INIT: k_mv<MV_INIT><<<g, kTile, 0, s>>>(v); break;
    case MV_STD_A: k_mv<MV_STD_A><<<g, kTile, 0, s>>>(v); break;
    case MV_CG_FIRST: k_mv<MV_CG_FIRST><<<g, kTile, 0, s>>>(v); break;
    case MV_CG1: k_mv<MV_CG1><<<g, kTile, 0, s>>>(v); break;
    default: k_mv<MV_CHECK><<<g, kTile, 0, s>>>(v); break;
  }
}
void launch_std_update(bool check, const DevView& v, cudaStream_t s) {
  if (check) k_std_update<true><<<tile_grid(v), kTile, 0, s>>>(v);
  else k_std_update<false><<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_cg_first_update(const DevView& v, cudaStream_t s) {
  k_cg_first_update<<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_cg_update(bool check, const DevView& v, cudaStream_t s) {
  if (check) k_cg_update<true><<<tile_grid(v), kTile, 0, s>>>(v);
  else k_cg_update<false><<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_picard_check(const DevView& v, cudaStream_t s) {
  k_picard_check<<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_mixed_setup(const DevView& v, cudaStream_t s) {
  k_scale<<<tile_grid(v), kTile, 0, s>>>(v);
  k_make_a32<<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_refine_resid(const DevView& v, cudaStream_t s) {
  k_refine_resid<<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_inner_a(const DevView& v, cudaStream_t s) { k_inner_a<<<tile_grid(v), kTile, 0, s>>>(v); }
void launch_inner_b(const DevView& v, cudaStream_t s) { k_inner_b<<<tile_grid(v), kTile, 0, s>>>(v); }
void launch_inner(const DevView& v, cudaStream_t s) {
  launch_inner_a(v, s);
  launch_inner_b(v, s);
}
void launch_refine_update(const DevView& v, cudaStream_t s) {
  k_refine_update<<<tile_grid(v), kTile, 0, s>>>(v);
}
void launch_matvec_plain(const DevView& v, const double2* x, double2* y, cudaStream_t s) {
  k_matvec_plain<<<tile_grid(v), kTile, 0, s>>>(v, x, y);
}
void launch_dinv(const DevView& v, int precond, cudaStream_t s) {
  k_dinv<<<tile_grid(v), kTile, 0, s>>>(v, precond);
}
void launch_bb(const DevView& v, cudaStream_t s) { k_bb<<<tile_grid(v), kTile, 0, s>>>(v); }

}  // namespace bp
