// bp_body.h -- per-thread arithmetic of the device kernels.
//
// Everything here is plain per-node / per-element arithmetic on a DevView,
// compiled as __host__ __device__ so the exact same code can also be checked
// against the CPU oracle without a GPU (tests/hostemu).  Block reductions,
// shuffles and launch logic live in bp_kernels.cu.
#pragma once

#include <cmath>

#include "bp_common.h"

#if defined(__CUDA_ARCH__)
#define BP_LD_STREAM(p) __ldcs(p)
#define BP_LD_RO(p) __ldg(p)
#define BP_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define BP_LD_STREAM(p) (*(p))
#define BP_LD_RO(p) (*(p))
#define BP_FMA(a, b, c) std::fma((a), (b), (c))
#endif

namespace bp {

// ---------------------------------------------------------------------
// Reference-element tables, glissade_velo_higher_init
// (glissade_velo_higher.F90:270-650).  Node numbering: 1-4 lower face
// (SW, SE, NE, NW), 5-8 upper face; quadrature points likewise at
// +-1/sqrt(3), unit weights.
// ---------------------------------------------------------------------
struct RefTables {
  double dxr[8][8], dyr[8][8], dzr[8][8];  // [p][n] d(phi_n)/d(xi) at point p
  double phi2[4][4];                        // [p][n] bilinear face basis
  double dxr2[4][4], dyr2[4][4];            // [p][n]
};

inline void fill_ref_tables(RefTables* t) {
  const double r = 1.0 / std::sqrt(3.0);
  const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  const double sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  const double sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int p = 0; p < 8; ++p) {
    const double x = sx[p] * r, y = sy[p] * r, z = sz[p] * r;
    for (int n = 0; n < 8; ++n) {
      t->dxr[p][n] = sx[n] * (1.0 + sy[n] * y) * (1.0 + sz[n] * z) / 8.0;
      t->dyr[p][n] = sy[n] * (1.0 + sx[n] * x) * (1.0 + sz[n] * z) / 8.0;
      t->dzr[p][n] = sz[n] * (1.0 + sx[n] * x) * (1.0 + sy[n] * y) / 8.0;
    }
  }
  for (int p = 0; p < 4; ++p) {
    const double x = sx[p] * r, y = sy[p] * r;
    for (int n = 0; n < 4; ++n) {
      t->phi2[p][n] = (1.0 + sx[n] * x) * (1.0 + sy[n] * y) / 4.0;
      t->dxr2[p][n] = sx[n] * (1.0 + sy[n] * y) / 4.0;
      t->dyr2[p][n] = sy[n] * (1.0 + sx[n] * x) / 4.0;
    }
  }
}

// ishift/jshift/kshift (glissade_velo_higher.F90:453-486): offset of node
// nc relative to node nr inside one element; nodes 0..3 lower, 4..7 upper.
BP_HD constexpr int node_di(int n) { return (n == 1 || n == 2 || n == 5 || n == 6) ? 1 : 0; }
BP_HD constexpr int node_dj(int n) { return (n == 2 || n == 3 || n == 6 || n == 7) ? 1 : 0; }
BP_HD constexpr int node_up(int n) { return n >= 4 ? 1 : 0; }
// stencil index (0-based indxA_3d) into which K(nr,nc) is summed; k grows downward
BP_HD constexpr int elem_m(int nr, int nc) {
  return (node_di(nc) - node_di(nr) + 1) + 3 * (node_dj(nc) - node_dj(nr) + 1) +
         9 * (node_up(nr) - node_up(nc) + 1);
}

// ---------------------------------------------------------------------
// Pass 1 of assembly: one quadrature point of one element.
// get_basis_function_derivatives_3d (:6360-6579) and
// compute_effective_viscosity (:7199-7378), in three pieces that the
// post-solve stress diagnostic shares.
// ---------------------------------------------------------------------
// J^-1 (row-major, Ji[3*row+col]) of the element's map at quadrature point
// p; false for a singular Jacobian.
BP_HD bool qp_jacobian_inverse(const RefTables& T, int p, const double* x, const double* y,
                               const double* z, double* Ji, double* det_out) {
  double J00 = 0, J01 = 0, J02 = 0, J10 = 0, J11 = 0, J12 = 0, J20 = 0, J21 = 0, J22 = 0;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const double a = T.dxr[p][n], b = T.dyr[p][n], c = T.dzr[p][n];
    J00 += a * x[n]; J01 += a * y[n]; J02 += a * z[n];
    J10 += b * x[n]; J11 += b * y[n]; J12 += b * z[n];
    J20 += c * x[n]; J21 += c * y[n]; J22 += c * z[n];
  }
  const double c00 = J11 * J22 - J12 * J21;
  const double c01 = -(J10 * J22 - J12 * J20);
  const double c02 = J10 * J21 - J11 * J20;
  const double c10 = -(J01 * J22 - J02 * J21);
  const double c11 = J00 * J22 - J02 * J20;
  const double c12 = -(J00 * J21 - J01 * J20);
  const double c20 = J01 * J12 - J02 * J11;
  const double c21 = -(J00 * J12 - J02 * J10);
  const double c22 = J00 * J11 - J01 * J10;
  const double det = J00 * c00 + J01 * c01 + J02 * c02;
  *det_out = det;
  if (!(fabs(det) > 0.0)) return false;
  // Jinv(row,col) = cofactor(col,row)/detJ
  Ji[0] = c00 / det; Ji[1] = c10 / det; Ji[2] = c20 / det;
  Ji[3] = c01 / det; Ji[4] = c11 / det; Ji[5] = c21 / det;
  Ji[6] = c02 / det; Ji[7] = c12 / det; Ji[8] = c22 / det;
  return true;
}

// Velocity gradient at quadrature point p: g = (du/dx, du/dy, du/dz,
// dv/dx, dv/dy, dv/dz), the derivatives of the basis functions formed from
// J^-1 in one fixed fma pattern.
BP_HD void qp_velocity_gradient(const RefTables& T, int p, const double* Ji, const double* u,
                                const double* w, double* g) {
  double ux = 0, uy = 0, uz = 0, vx = 0, vy = 0, vz = 0;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const double a = T.dxr[p][n], b = T.dyr[p][n], c = T.dzr[p][n];
    const double dx = BP_FMA(Ji[2], c, BP_FMA(Ji[1], b, Ji[0] * a));
    const double dy = BP_FMA(Ji[5], c, BP_FMA(Ji[4], b, Ji[3] * a));
    const double dz = BP_FMA(Ji[8], c, BP_FMA(Ji[7], b, Ji[6] * a));
    ux += dx * u[n]; uy += dy * u[n]; uz += dz * u[n];
    vx += dx * w[n]; vy += dy * w[n]; vz += dz * w[n];
  }
  g[0] = ux; g[1] = uy; g[2] = uz; g[3] = vx; g[4] = vy; g[5] = vz;
}

// compute_effective_viscosity, 3-D higher-order branch: constant, from the
// flow factor at a fixed strain rate, or Glen's law (n = 3) with the
// 1e-8 /a strain-rate floor; g is read only by the last.
BP_HD double qp_efvs(int which_efvs, double efvs_constant, double flwafact, const double* g) {
  if (which_efvs == 0) return efvs_constant;
  if (which_efvs == 1) {
    const double scyr = 31536000.0;
    const double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    return flwafact * pow(effstrain, (1.0 - 3.0) / 3.0);
  }
  const double ux = g[0], uy = g[1], uz = g[2], vx = g[3], vy = g[4], vz = g[5];
  const double smin = 1.0e-8;
  const double sq = smin * smin + (ux * ux + vy * vy + ux * vy + 0.25 * ((vx + uy) * (vx + uy))) +
                    0.25 * (uz * uz + vz * vz);
  const double p2 = ((1.0 - 3.0) / 3.0) / 2.0;
  return flwafact * pow(sq, p2);
}

// Writes f = efvs*w*detJ/vol0 and J^-1 (row-major) to out[0..9]; returns
// false for a singular Jacobian.
BP_HD bool qp_compute(const RefTables& T, int p, const double* x,
                      const double* y, const double* z, const double* u,
                      const double* w, int which_efvs, double efvs_constant,
                      double flwafact, double* out, double* efvs_qp) {
  double Ji[9], det;
  if (!qp_jacobian_inverse(T, p, x, y, z, Ji, &det)) return false;
  double g[6] = {0, 0, 0, 0, 0, 0};
  if (which_efvs == 2) qp_velocity_gradient(T, p, Ji, u, w, g);
  const double efvs = qp_efvs(which_efvs, efvs_constant, flwafact, g);
  *efvs_qp = efvs;
  out[0] = efvs * 1.0 * det / kVol0;
#pragma unroll
  for (int i = 0; i < 9; ++i) out[1 + i] = Ji[i];
  return true;
}

// The 8 nodes of element e (cell, layer kk): coordinates and velocity
// (zero at a corner without a column); returns the element's instance.
BP_HD const InstParams& elem_gather(const DevView& v, int e, double* x, double* y, double* z,
                                    double* u, double* w) {
  const int nz = v.nz, nl = nz - 1;
  const int cell = e / nl, kk = e - cell * nl;
  const InstParams& ip = v.inst[v.cell_inst[cell]];
  const int ic = v.cell_ij[cell], jc = v.cell_ij[v.ncells + cell];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const int corner = n & 3;              // SW, SE, NE, NW
    const int lev = n < 4 ? kk + 1 : kk;   // nodes 1-4 lower (k+1), 5-8 upper (k)
    const int iv = (corner == 1 || corner == 2) ? ic : ic - 1;
    const int jv = (corner >= 2) ? jc : jc - 1;
    x[n] = ip.dx * iv;
    y[n] = ip.dy * jv;
    const double s = v.cell_s[corner * v.ncells + cell];
    const double h = v.cell_h[corner * v.ncells + cell];
    z[n] = s - ip.sigma[lev] * h;
    const int col = v.cell_cols[corner * v.ncells + cell];
    if (col >= 0) {
      const double2 xv = v.x[node_of(v, col, lev)];
      u[n] = xv.x; w[n] = xv.y;
    } else {
      u[n] = 0.0; w[n] = 0.0;
    }
  }
  return ip;
}

// Gather the 8 nodes of element e and run qp_compute.
BP_HD bool qp_element_point(const DevView& v, const RefTables& T, int e, int p,
                            double* out, double* efvs_qp) {
  double x[8], y[8], z[8], u[8], w[8];
  const InstParams& ip = elem_gather(v, e, x, y, z, u, w);
  return qp_compute(T, p, x, y, z, u, w, ip.which_efvs, ip.efvs_constant,
                    v.flwafact[e], out, efvs_qp);
}

// compute_internal_stress (:6968-7195) for element e at the current 3-D
// velocity: the velocity gradient and the effective viscosity at the 8
// quadrature points (assembly's arithmetic), tau_xz = efvs du/dz, tau_yz =
// efvs dv/dz, tau_xx = 2 efvs du/dx, tau_yy = 2 efvs dv/dy, tau_xy = efvs
// (dv/dx + du/dy), each averaged, and tau_eff from the averages.  The
// shallow-shelf solve takes the horizontal gradients only and its
// viscosity branch (:7110-7116, :7325-7338); L1L2 takes the element's
// layer viscosity v.efvs[e] at every point (:7135-7139); Blatter-Pattyn
// and DIVA the 3-D gradients and viscosity.  tau = {xz, yz, xx, yy, xy,
// eff}; false for a singular Jacobian.
BP_HD bool stress_element(const DevView& v, const RefTables& T, int e, double* tau) {
  double x[8], y[8], z[8], u[8], w[8];
  const InstParams& ip = elem_gather(v, e, x, y, z, u, w);
  double txz = 0.0, tyz = 0.0, txx = 0.0, tyy = 0.0, txy = 0.0;
  for (int p = 0; p < 8; ++p) {
    double Ji[9], det, g[6];
    if (!qp_jacobian_inverse(T, p, x, y, z, Ji, &det)) return false;
    qp_velocity_gradient(T, p, Ji, u, w, g);
    if (v.solve2d && !v.l1l2 && !v.diva) {
      g[2] = 0.0;
      g[5] = 0.0;
    }
    const double efvs = v.l1l2 ? v.efvs[e] : qp_efvs(ip.which_efvs, ip.efvs_constant, v.flwafact[e], g);
    txz = txz + efvs * g[2];
    tyz = tyz + efvs * g[5];
    txx = txx + 2.0 * efvs * g[0];
    tyy = tyy + 2.0 * efvs * g[4];
    txy = txy + efvs * (g[3] + g[1]);
  }
  txz = txz / 8; tyz = tyz / 8; txx = txx / 8; tyy = tyy / 8; txy = txy / 8;
  tau[0] = txz; tau[1] = tyz; tau[2] = txx; tau[3] = tyy; tau[4] = txy;
  tau[5] = sqrt(txx * txx + tyy * tyy + txx * tyy + txy * txy + txz * txz + tyz * tyz);
  return true;
}

// compute_basal_friction_heatflx (:6755-6964): the frictional heat flux
// beta |u_b|^2 / scyr (W/m^2).  Finite-element method (which = 0), one
// active cell: the corner values (bed velocity, zero at a corner without a
// column; corner beta) interpolated to the 4 face quadrature points, the
// weighted mean of beta |u|^2 (:6853-6887).  Local method (which = 1), one
// column: beta |u_b|^2 at the vertex (:6900-6909), unstaggered to the cells
// on the way out.
BP_HD double bfric_cell(const DevView& v, const RefTables& T, int cell) {
  const int nz = v.nz;
  double u[4], w[4], b[4];
  for (int q = 0; q < 4; ++q) {  // SW, SE, NE, NW = the reference's 2-D node order
    const int col = v.cell_cols[q * v.ncells + cell];
    if (col >= 0) {
      const double2 xb = v.x[node_of(v, col, nz - 1)];
      u[q] = xb.x;
      w[q] = xb.y;
    } else {
      u[q] = 0.0;
      w[q] = 0.0;
    }
    b[q] = v.cell_beta[q * v.ncells + cell];
  }
  double f = 0.0, sum_w = 0.0;
  for (int p = 0; p < 4; ++p) {
    double uq = 0.0, vq = 0.0, bq = 0.0;
    for (int n = 0; n < 4; ++n) {
      uq = uq + T.phi2[p][n] * u[n];
      vq = vq + T.phi2[p][n] * w[n];
      bq = bq + T.phi2[p][n] * b[n];
    }
    f = f + 1.0 * bq * (uq * uq + vq * vq);  // wqp_2d = 1
    sum_w = sum_w + 1.0;
  }
  return f / (sum_w * 31536000.0);
}

BP_HD double bfric_vertex(const DevView& v, int col) {
  const double2 xb = v.x[node_of(v, col, v.nz - 1)];
  return v.col_beta[col] * (xb.x * xb.x + xb.y * xb.y) / 31536000.0;
}

// ---------------------------------------------------------------------
// Pass 2 of assembly: the row of node (col,k) in block B (0 uu, 1 uv,
// 2 vu, 3 vv), gathered from its incident elements in the reference's
// element order (j, then i, then k).  compute_element_matrix (:7868-7986)
// and element_to_global_matrix_3d (:7990-8054).  The element terms use
// one fixed fma pattern so that K(nr,nc) and K(nc,nr) are bitwise equal
// and the assembled matrix is exactly symmetric.
// ---------------------------------------------------------------------
template <int B>
BP_HD double block_term(double ar, double br, double cr, double ac, double bc, double cc) {
  if (B == 0) return BP_FMA(cr, cc, BP_FMA(4.0 * ar, ac, br * bc));
  if (B == 1) return BP_FMA(2.0 * ar, bc, br * ac);
  if (B == 2) return BP_FMA(2.0 * br, ac, ar * bc);
  return BP_FMA(cr, cc, BP_FMA(4.0 * br, bc, ar * ac));
}

template <int NR, int B>
BP_HD void row_element(const RefTables& T, const double* qpe, double* acc) {
  double K[8];
#pragma unroll
  for (int nc = 0; nc < 8; ++nc) K[nc] = 0.0;
  for (int p = 0; p < 8; ++p) {
    const double* q = qpe + p * 10;
    const double f = BP_LD_RO(q + 0);
    const double i00 = BP_LD_RO(q + 1), i01 = BP_LD_RO(q + 2), i02 = BP_LD_RO(q + 3);
    const double i10 = BP_LD_RO(q + 4), i11 = BP_LD_RO(q + 5), i12 = BP_LD_RO(q + 6);
    const double i20 = BP_LD_RO(q + 7), i21 = BP_LD_RO(q + 8), i22 = BP_LD_RO(q + 9);
    double ax[8], ay[8], az[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const double a = T.dxr[p][n], b = T.dyr[p][n], c = T.dzr[p][n];
      ax[n] = BP_FMA(i02, c, BP_FMA(i01, b, i00 * a));
      ay[n] = BP_FMA(i12, c, BP_FMA(i11, b, i10 * a));
      az[n] = BP_FMA(i22, c, BP_FMA(i21, b, i20 * a));
    }
#pragma unroll
    for (int nc = 0; nc < 8; ++nc)
      K[nc] = BP_FMA(f, block_term<B>(ax[NR], ay[NR], az[NR], ax[nc], ay[nc], az[nc]), K[nc]);
  }
#pragma unroll
  for (int nc = 0; nc < 8; ++nc) acc[elem_m(NR, nc)] += K[nc];
}

// Element index of (cell, layer) or -1.
BP_HD int elem_of(int cell, int kk, int nz) { return cell < 0 ? -1 : cell * (nz - 1) + kk; }

template <int B>
BP_HD void row_assemble(const DevView& v, const RefTables& T, int col, int k,
                        double* acc) {
  const int nz = v.nz, nc = v.ncols;
#pragma unroll
  for (int m = 0; m < 27; ++m) acc[m] = 0.0;
  const int c0 = v.col_cells[0 * nc + col];  // cell (i,j):     vertex is its NE corner
  const int c1 = v.col_cells[1 * nc + col];  // cell (i+1,j):   NW corner
  const int c2 = v.col_cells[2 * nc + col];  // cell (i,j+1):   SE corner
  const int c3 = v.col_cells[3 * nc + col];  // cell (i+1,j+1): SW corner
  const bool lo = k >= 1, up = k <= nz - 2;  // element above (k-1) / below (k)
  const double* qp = v.qp;
  if (c0 >= 0) {
    if (lo) row_element<2, B>(T, qp + (size_t)elem_of(c0, k - 1, nz) * 80, acc);
    if (up) row_element<6, B>(T, qp + (size_t)elem_of(c0, k, nz) * 80, acc);
  }
  if (c1 >= 0) {
    if (lo) row_element<3, B>(T, qp + (size_t)elem_of(c1, k - 1, nz) * 80, acc);
    if (up) row_element<7, B>(T, qp + (size_t)elem_of(c1, k, nz) * 80, acc);
  }
  if (c2 >= 0) {
    if (lo) row_element<1, B>(T, qp + (size_t)elem_of(c2, k - 1, nz) * 80, acc);
    if (up) row_element<5, B>(T, qp + (size_t)elem_of(c2, k, nz) * 80, acc);
  }
  if (c3 >= 0) {
    if (lo) row_element<0, B>(T, qp + (size_t)elem_of(c3, k - 1, nz) * 80, acc);
    if (up) row_element<4, B>(T, qp + (size_t)elem_of(c3, k, nz) * 80, acc);
  }
}

// Element-centric form of pass 2, in two steps with row_element's
// arithmetic regrouped.  element_row_blocks: row nr (a corner, 0..7) of an
// element's four 8 x 8 blocks, K[B * 8 + nc], each entry accumulated over
// the quadrature points in order with row_element's operations, so that it
// is bitwise the value row_element adds; the physical basis gradients of a
// point are formed once for all four blocks.  row_gather: the row of node
// (col,k) in block B, summed from the stored element rows in
// row_assemble's element order, so the assembled row is bitwise
// row_assemble's.  Ke holds [element][B][nr][nc].
BP_HD void element_row_blocks(const RefTables& T, const double* qpe, int nr, double* K) {
#pragma unroll
  for (int i = 0; i < 32; ++i) K[i] = 0.0;
  for (int p = 0; p < 8; ++p) {
    const double* q = qpe + p * 10;
    const double f = BP_LD_RO(q + 0);
    const double i00 = BP_LD_RO(q + 1), i01 = BP_LD_RO(q + 2), i02 = BP_LD_RO(q + 3);
    const double i10 = BP_LD_RO(q + 4), i11 = BP_LD_RO(q + 5), i12 = BP_LD_RO(q + 6);
    const double i20 = BP_LD_RO(q + 7), i21 = BP_LD_RO(q + 8), i22 = BP_LD_RO(q + 9);
    const double ar = T.dxr[p][nr], br = T.dyr[p][nr], cr = T.dzr[p][nr];
    const double axr = BP_FMA(i02, cr, BP_FMA(i01, br, i00 * ar));
    const double ayr = BP_FMA(i12, cr, BP_FMA(i11, br, i10 * ar));
    const double azr = BP_FMA(i22, cr, BP_FMA(i21, br, i20 * ar));
#pragma unroll
    for (int nc = 0; nc < 8; ++nc) {
      const double a = T.dxr[p][nc], b = T.dyr[p][nc], c = T.dzr[p][nc];
      const double ax = BP_FMA(i02, c, BP_FMA(i01, b, i00 * a));
      const double ay = BP_FMA(i12, c, BP_FMA(i11, b, i10 * a));
      const double az = BP_FMA(i22, c, BP_FMA(i21, b, i20 * a));
      K[nc] = BP_FMA(f, block_term<0>(axr, ayr, azr, ax, ay, az), K[nc]);
      K[8 + nc] = BP_FMA(f, block_term<1>(axr, ayr, azr, ax, ay, az), K[8 + nc]);
      K[16 + nc] = BP_FMA(f, block_term<2>(axr, ayr, azr, ax, ay, az), K[16 + nc]);
      K[24 + nc] = BP_FMA(f, block_term<3>(axr, ayr, azr, ax, ay, az), K[24 + nc]);
    }
  }
}

template <int NR, int B>
BP_HD void gather_element(const double* Ke, int e, double* acc) {
  const double* r = Ke + ((size_t)e * 4 + B) * 64 + NR * 8;
#pragma unroll
  for (int nc = 0; nc < 8; ++nc) acc[elem_m(NR, nc)] += BP_LD_RO(r + nc);
}

template <int B>
BP_HD void row_gather(const DevView& v, const double* Ke, int col, int k, double* acc) {
  const int nz = v.nz, nc = v.ncols;
#pragma unroll
  for (int m = 0; m < 27; ++m) acc[m] = 0.0;
  const int c0 = v.col_cells[0 * nc + col], c1 = v.col_cells[1 * nc + col];
  const int c2 = v.col_cells[2 * nc + col], c3 = v.col_cells[3 * nc + col];
  const bool lo = k >= 1, up = k <= nz - 2;
  if (c0 >= 0) {
    if (lo) gather_element<2, B>(Ke, elem_of(c0, k - 1, nz), acc);
    if (up) gather_element<6, B>(Ke, elem_of(c0, k, nz), acc);
  }
  if (c1 >= 0) {
    if (lo) gather_element<3, B>(Ke, elem_of(c1, k - 1, nz), acc);
    if (up) gather_element<7, B>(Ke, elem_of(c1, k, nz), acc);
  }
  if (c2 >= 0) {
    if (lo) gather_element<1, B>(Ke, elem_of(c2, k - 1, nz), acc);
    if (up) gather_element<5, B>(Ke, elem_of(c2, k, nz), acc);
  }
  if (c3 >= 0) {
    if (lo) gather_element<0, B>(Ke, elem_of(c3, k - 1, nz), acc);
    if (up) gather_element<4, B>(Ke, elem_of(c3, k, nz), acc);
  }
}

// ---------------------------------------------------------------------
// Shallow-shelf (SSA) assembly: assemble_stiffness_matrix_2d, SSA branch
// (:5208-5595).  One 2-D element per active cell (corners SW, SE, NE, NW =
// the reference's 2-D node order), 2x2 Gauss points; nodes are columns
// (nz = 1).  The element data of cell c sit where the 3-D elements' do:
// point p at qp[(c * 8 + p) * 10], f then J^-1 (2 x 2, row-major).
// ---------------------------------------------------------------------
// compute_effective_viscosity_L1L2 (:7382-7618): the viscosity ek[k] of
// each layer k = 0..nl-1 at one point, from the strain rates g (as
// qp_velocity_gradient), the surface slope (sx, sy) and the thickness h
// there.  Glen's law (n = 3) solves x^3 + a x + b = 0 for x =
// tau_parallel, a = tau_perp^2 = (rhoi grav h sigma(k+1) |grad s|)^2 and
// b = -effstrain / A, by Cardano's formula (:7566-7600), the second root
// in its first-order form -a / (3 |b|^(1/3)) when a^3/27 <= 1e-6 b^2/4;
// efvs = 1 / (2 A (x^2 + tau_perp^2)).  Returns the column average
// sum_k ek[k] (sigma(k+1) - sigma(k)) (:5474-5478).
BP_HD double l1l2_point_efvs(const InstParams& ip, int nl, const double* flwa, const double* flwafact,
                             const double* g, double sx, double sy, double h, double* ek) {
  if (ip.which_efvs == 0) {
    for (int k = 0; k < nl; ++k) ek[k] = ip.efvs_constant;
  } else if (ip.which_efvs == 1) {
    const double scyr = 31536000.0;
    const double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    for (int k = 0; k < nl; ++k) ek[k] = flwafact[k] * pow(effstrain, (1.0 - 3.0) / 3.0);
  } else {
    const double ux = g[0], uy = g[1], vx = g[3], vy = g[4];
    const double smin = 1.0e-8;
    const double effstrain = sqrt(smin * smin + ux * ux + vy * vy + ux * vy + 0.25 * ((vx + uy) * (vx + uy)));
    const double grads = sqrt(sx * sx + sy * sy);
    for (int k = 0; k < nl; ++k) {
      const double tau_perp = ip.rhoi * ip.grav * (h * ip.sigma[k + 1]) * grads;
      const double a = tau_perp * tau_perp;
      const double b = -effstrain / flwa[k];
      const double a3 = a * a * a / 27.0, b2 = b * b / 4.0;
      const double c = sqrt(b2 + a3);
      const double rootA = pow(-b / 2.0 + c, 1.0 / 3.0);
      const double rootB = a3 > 1.0e-6 * b2 ? -pow(b / 2.0 + c, 1.0 / 3.0) : -a / (3.0 * pow(fabs(b), 1.0 / 3.0));
      const double tp = rootA + rootB;
      ek[k] = 1.0 / (2.0 * flwa[k] * (tp * tp + tau_perp * tau_perp));
    }
  }
  double avg = 0.0;
  for (int k = 0; k < nl; ++k) avg = avg + ek[k] * (ip.sigma[k + 1] - ip.sigma[k]);
  return avg;
}

// compute_effective_viscosity_diva (:7622-7864), the default non-cubic
// form: the viscosity of each layer k at one point from the horizontal
// strain rates g of the mean velocity and the vertical shear (du/dz,
// dv/dz) = (taux, tauy) stagsigma(k) / efvs_old(k), (taux, tauy) the basal
// traction at the point.  ek: in the last assembly's values (0 = none yet:
// the value at the 1e-8 /a strain-rate floor), out the new ones.  Returns
// the column average sum_k ek[k] (sigma(k+1) - sigma(k)).
BP_HD double diva_point_efvs(const InstParams& ip, int nl, const double* flwafact, const double* g,
                             double taux, double tauy, double* ek) {
  const double p_effstr = (1.0 - 3.0) / 3.0;
  if (ip.which_efvs == 0) {
    for (int k = 0; k < nl; ++k) ek[k] = ip.efvs_constant;
  } else if (ip.which_efvs == 1) {
    const double scyr = 31536000.0;
    const double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    for (int k = 0; k < nl; ++k) ek[k] = flwafact[k] * pow(effstrain, p_effstr);
  } else {
    const double ux = g[0], uy = g[1], vx = g[3], vy = g[4];
    const double smin = 1.0e-8;
    for (int k = 0; k < nl; ++k) {
      if (ek[k] == 0.0) ek[k] = flwafact[k] * pow(smin, p_effstr);
      const double stagsigma = (ip.sigma[k] + ip.sigma[k + 1]) / 2.0;
      const double du_dz = taux * stagsigma / ek[k];
      const double dv_dz = tauy * stagsigma / ek[k];
      const double sq = smin * smin + ux * ux + vy * vy + ux * vy + 0.25 * ((vx + uy) * (vx + uy)) +
                        0.25 * (du_dz * du_dz + dv_dz * dv_dz);
      ek[k] = flwafact[k] * pow(sq, p_effstr / 2);
    }
  }
  double avg = 0.0;
  for (int k = 0; k < nl; ++k) avg = avg + ek[k] * (ip.sigma[k + 1] - ip.sigma[k]);
  return avg;
}

// Point p of cell c: get_basis_function_derivatives_2d (:6583-6751); the
// shallow-shelf branch of compute_effective_viscosity with the vertically
// averaged flow factor (v.flwafact[c]), or the L1L2 or DIVA layer
// viscosities (written to ek; DIVA also updates v.eq3) and their column
// average; f = h efvs w detJ / vol0 with the thickness interpolated to the
// point (:5507-5515, compute_element_matrix :7868-7986).  false for a
// singular Jacobian.
BP_HD bool qp2_element_point(const DevView& v, const RefTables& T, int c, int p, double* out,
                             double* efvs_qp, double* ek = nullptr) {
  const InstParams& ip = v.inst[v.cell_inst[c]];
  const int ic = v.cell_ij[c], jc = v.cell_ij[v.ncells + c];
  double x[4], y[4], u[4], w[4], h[4];
  for (int n = 0; n < 4; ++n) {
    const int iv = (n == 1 || n == 2) ? ic : ic - 1;
    const int jv = n >= 2 ? jc : jc - 1;
    x[n] = ip.dx * iv;
    y[n] = ip.dy * jv;
    h[n] = v.cell_h[n * v.ncells + c];
    const int col = v.cell_cols[n * v.ncells + c];
    if (col >= 0) {
      const double2 xv = v.x[v.col_node[col]];
      u[n] = xv.x;
      w[n] = xv.y;
    } else {
      u[n] = 0.0;
      w[n] = 0.0;
    }
  }
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
  for (int n = 0; n < 4; ++n) {
    J11 += T.dxr2[p][n] * x[n];
    J12 += T.dxr2[p][n] * y[n];
    J21 += T.dyr2[p][n] * x[n];
    J22 += T.dyr2[p][n] * y[n];
  }
  const double det = J11 * J22 - J12 * J21;
  if (!(fabs(det) > 0.0)) return false;
  const double i11 = J22 / det, i12 = -J12 / det, i21 = -J21 / det, i22 = J11 / det;
  double g[6] = {0, 0, 0, 0, 0, 0};  // (du/dx, du/dy, -, dv/dx, dv/dy, -)
  if (ip.which_efvs == 2) {
    for (int n = 0; n < 4; ++n) {
      const double dx = BP_FMA(i12, T.dyr2[p][n], i11 * T.dxr2[p][n]);
      const double dy = BP_FMA(i22, T.dyr2[p][n], i21 * T.dxr2[p][n]);
      g[0] += dx * u[n];
      g[1] += dy * u[n];
      g[3] += dx * w[n];
      g[4] += dy * w[n];
    }
  }
  double h_qp = 0.0;
  for (int n = 0; n < 4; ++n) h_qp += T.phi2[p][n] * h[n];
  double efvs;
  if (v.l1l2) {
    const int nl = v.nl;
    double sx = 0.0, sy = 0.0;
    for (int n = 0; n < 4; ++n) {
      sx += T.phi2[p][n] * v.cell_ds[(size_t)n * v.ncells + c];
      sy += T.phi2[p][n] * v.cell_ds[(size_t)(4 + n) * v.ncells + c];
    }
    efvs = l1l2_point_efvs(ip, nl, v.cell_flwa + (size_t)c * nl, v.flwafact + (size_t)c * nl, g, sx, sy, h_qp,
                           ek);
  } else if (v.diva) {
    // basal traction at the point from the corners' columns (zero outside
    // an outflow domain, where beta_eff is zero)
    const int nl = v.nl;
    double taux = 0.0, tauy = 0.0;
    for (int n = 0; n < 4; ++n) {
      const int col = v.cell_cols[n * v.ncells + c];
      taux += T.phi2[p][n] * (col >= 0 ? v.col_bt[col].x : 0.0);
      tauy += T.phi2[p][n] * (col >= 0 ? v.col_bt[col].y : 0.0);
    }
    double* e3 = v.eq3 + ((size_t)c * 4 + p) * nl;
    for (int k = 0; k < nl; ++k) ek[k] = e3[k];
    efvs = diva_point_efvs(ip, nl, v.flwafact + (size_t)c * nl, g, taux, tauy, ek);
    for (int k = 0; k < nl; ++k) e3[k] = ek[k];
  } else {
    // qp_efvs with no vertical shear is the SSA branch (:7326-7334)
    efvs = qp_efvs(ip.which_efvs, ip.efvs_constant, v.flwafact[c], g);
  }
  *efvs_qp = efvs;
  out[0] = h_qp * efvs * 1.0 * det / kVol0;
  out[1] = i11; out[2] = i12; out[3] = i21; out[4] = i22;
  return true;
}

// stencil index (0-based, kA = 0) into which the 2-D K(nr, nc) is summed
BP_HD constexpr int elem_m2(int nr, int nc) {
  return (node_di(nc) - node_di(nr) + 1) + 3 * (node_dj(nc) - node_dj(nr) + 1) + 9;
}

// Row NR of the 2-D element matrix in block B (the SSA terms of
// compute_element_matrix: block_term without the vertical ones).
template <int NR, int B>
BP_HD void row_element2(const RefTables& T, const double* qpe, double* acc) {
  double K[4] = {0.0, 0.0, 0.0, 0.0};
  for (int p = 0; p < 4; ++p) {
    const double* q = qpe + p * 10;
    const double f = BP_LD_RO(q + 0);
    const double i11 = BP_LD_RO(q + 1), i12 = BP_LD_RO(q + 2), i21 = BP_LD_RO(q + 3), i22 = BP_LD_RO(q + 4);
    double ax[4], ay[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      ax[n] = BP_FMA(i12, T.dyr2[p][n], i11 * T.dxr2[p][n]);
      ay[n] = BP_FMA(i22, T.dyr2[p][n], i21 * T.dxr2[p][n]);
    }
#pragma unroll
    for (int nc = 0; nc < 4; ++nc)
      K[nc] = BP_FMA(f, block_term<B>(ax[NR], ay[NR], 0.0, ax[nc], ay[nc], 0.0), K[nc]);
  }
#pragma unroll
  for (int nc = 0; nc < 4; ++nc) acc[elem_m2(NR, nc)] += K[nc];
}

// The row of column col in block B gathered from its incident cells in the
// reference's element order (element_to_global_matrix_2d :8058-8121).
template <int B>
BP_HD void row_assemble2(const DevView& v, const RefTables& T, int col, double* acc) {
  const int nc = v.ncols;
#pragma unroll
  for (int m = 0; m < 27; ++m) acc[m] = 0.0;
  const int c0 = v.col_cells[0 * nc + col];  // the vertex is the NE corner of c0,
  const int c1 = v.col_cells[1 * nc + col];  // NW of c1, SE of c2, SW of c3
  const int c2 = v.col_cells[2 * nc + col];
  const int c3 = v.col_cells[3 * nc + col];
  if (c0 >= 0) row_element2<2, B>(T, v.qp + (size_t)c0 * 80, acc);
  if (c1 >= 0) row_element2<3, B>(T, v.qp + (size_t)c1 * 80, acc);
  if (c2 >= 0) row_element2<1, B>(T, v.qp + (size_t)c2 * 80, acc);
  if (c3 >= 0) row_element2<0, B>(T, v.qp + (size_t)c3 * 80, acc);
}

// ---------------------------------------------------------------------
// L1L2 3-D velocity: compute_3d_velocity_L1L2 (:5834-6356), the vertex
// method (edge_velocity = .false.), after the Picard loop.
// ---------------------------------------------------------------------
// Cell c: the strain rates of the basal velocity at the cell centre
// (get_basis_function_derivatives_2d with the centre derivatives
// :589-597), eps_parallel, and per layer k tau_parallel = 2 efvs
// eps_parallel and w1..w3 = E_k (2 ux + vy, uy + vx, 2 vy + ux), E_k the
// integral of efvs from the surface to the base of layer k; written to
// v.lw[(q * nl + k) * ncells + c], q = 0 tau_parallel, 1..3 w1..w3.
BP_HD void l1l2_cell(const DevView& v, int c) {
  const InstParams& ip = v.inst[v.cell_inst[c]];
  const int ic = v.cell_ij[c], jc = v.cell_ij[v.ncells + c], nl = v.nl;
  const double dxr[4] = {-0.25, 0.25, 0.25, -0.25}, dyr[4] = {-0.25, -0.25, 0.25, 0.25};
  double x[4], y[4], u[4], w[4];
  for (int n = 0; n < 4; ++n) {
    const int iv = (n == 1 || n == 2) ? ic : ic - 1;
    const int jv = n >= 2 ? jc : jc - 1;
    x[n] = ip.dx * iv;
    y[n] = ip.dy * jv;
    const int col = v.cell_cols[n * v.ncells + c];
    u[n] = col >= 0 ? v.x[v.col_node[col]].x : 0.0;
    w[n] = col >= 0 ? v.x[v.col_node[col]].y : 0.0;
  }
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
  for (int n = 0; n < 4; ++n) {
    J11 += dxr[n] * x[n];
    J12 += dxr[n] * y[n];
    J21 += dyr[n] * x[n];
    J22 += dyr[n] * y[n];
  }
  const double det = J11 * J22 - J12 * J21;
  double ux = 0.0, uy = 0.0, vx = 0.0, vy = 0.0;
  if (fabs(det) > 0.0) {
    const double i11 = J22 / det, i12 = -J12 / det, i21 = -J21 / det, i22 = J11 / det;
    for (int n = 0; n < 4; ++n) {
      const double dx = i11 * dxr[n] + i12 * dyr[n];
      const double dy = i21 * dxr[n] + i22 * dyr[n];
      ux += dx * u[n];
      uy += dy * u[n];
      vx += dx * w[n];
      vy += dy * w[n];
    }
  }
  const double eps = sqrt(ux * ux + vy * vy + ux * vy + 0.25 * ((vx + uy) * (vx + uy)));
  const double H = v.cell_thck[c];
  const size_t NC = (size_t)v.ncells, st = (size_t)nl * NC;
  double E = 0.0;
  for (int k = 0; k < nl; ++k) {
    const double e = v.efvs[(size_t)c * nl + k];
    E = E + e * (ip.sigma[k + 1] - ip.sigma[k]) * H;
    const size_t o = (size_t)k * NC + c;
    v.lw[o] = 2.0 * e * eps;
    v.lw[st + o] = E * (2.0 * ux + vy);
    v.lw[2 * st + o] = E * (uy + vx);
    v.lw[3 * st + o] = E * (2.0 * vy + ux);
  }
}

// glissade_gradient with gradient_margin = 1 (glissade_grid_operators.F90:
// 235-410) at a vertex: the mean of the two edge differences (a, b) whose
// cells both hold ice, the one such edge, or zero.
BP_HD double l1l2_edges(double a, double b, bool ma, bool mb) {
  if (ma && mb) return (a + b) / 2.0;
  if (ma) return a;
  if (mb) return b;
  return 0.0;
}

// Column col: per layer k from the bed up, tau_xz, tau_yz at the layer
// midpoint (the shallow-ice stress -rhoi grav depth grad s plus the
// gradients of w1..w3 over the four cells), A and tau_parallel staggered
// over the ice cells (glissade_stagger margin 1, NW NE SW SE), and u(k) =
// u(k+1) + 2 A tau_eff^2 (sigma(k+1) - sigma(k)) H tau_xz (tau_eff^(n-1)
// with n = 3); a prescribed basal vertex keeps the basal velocity on every
// level.  Writes v.x3[col * (nl + 1) + k], k = nl the bed.
BP_HD void l1l2_column(const DevView& v, int col) {
  const InstParams& ip = v.inst[v.col_inst[col]];
  const int nl = v.nl, nc = v.ncols;
  const size_t NCELL = (size_t)v.ncells, st = (size_t)nl * NCELL;
  // cells SW (i,j), SE (i+1,j), NW (i,j+1), NE (i+1,j+1)
  const int cs[4] = {v.col_cells[col], v.col_cells[nc + col], v.col_cells[2 * nc + col],
                     v.col_cells[3 * nc + col]};
  const bool sw = cs[0] >= 0, se = cs[1] >= 0, nw = cs[2] >= 0, ne = cs[3] >= 0;
  const double sx = v.col_ds[col], sy = v.col_ds[nc + col], H = v.col_h[col];
  const uint8_t dm = v.dmask[v.col_node[col]];
  const double2 ub = v.x[v.col_node[col]];
  double2* out = v.x3 + (size_t)col * (nl + 1);
  out[nl] = ub;
  double2 up = ub;
  for (int k = nl - 1; k >= 0; --k) {
    double f[4][4];  // [quantity][cell]
    for (int q = 0; q < 4; ++q)
      for (int m = 0; m < 4; ++m) f[q][m] = cs[m] >= 0 ? v.lw[q * st + (size_t)k * NCELL + cs[m]] : 0.0;
    double d[3][2];
    for (int q = 0; q < 3; ++q) {
      const double* g = f[q + 1];
      d[q][0] = l1l2_edges((g[3] - g[2]) / ip.dx, (g[1] - g[0]) / ip.dx, ne && nw, se && sw);
      d[q][1] = l1l2_edges((g[3] - g[1]) / ip.dy, (g[2] - g[0]) / ip.dy, ne && se, nw && sw);
    }
    const double depth = 0.5 * (ip.sigma[k] + ip.sigma[k + 1]) * H;
    const double txz = -ip.rhoi * ip.grav * depth * sx + 2.0 * d[0][0] + d[1][1];
    const double tyz = -ip.rhoi * ip.grav * depth * sy + d[1][0] + 2.0 * d[2][1];
    const int cnt = (int)nw + (int)ne + (int)sw + (int)se;
    double tp = 0.0, fa = 0.0;
    if (cnt > 0) {
      double a = 0.0, t = 0.0;
      const int order[4] = {2, 3, 0, 1};  // NW, NE, SW, SE
      for (int o = 0; o < 4; ++o) {
        const int m = order[o];
        if (cs[m] >= 0) {
          t = t + f[0][m];
          a = a + v.cell_flwa[(size_t)cs[m] * nl + k];
        }
      }
      tp = t / (double)cnt;
      fa = a / (double)cnt;
    }
    const double tes = tp * tp + txz * txz + tyz * tyz;
    const double fact = 2.0 * fa * tes * (ip.sigma[k + 1] - ip.sigma[k]) * H;
    double2 cur;
    cur.x = (dm & 1) ? ub.x : up.x + fact * txz;
    cur.y = (dm & 2) ? ub.y : up.y + fact * tyz;
    out[k] = cur;
    up = cur;
  }
}

// ---------------------------------------------------------------------
// DIVA (Goldberg 2011): omega, beta_eff and the 3-D velocity.
// ---------------------------------------------------------------------
// compute_integrals_diva (:5601-5726) of cell c from its point viscosities
// v.eq3: per point the integral of depth / efvs from the bed up to each
// level, averaged over the points (omega_k, over H), and its
// layer-midpoint integral over the column (omega, over H).
BP_HD void diva_cell_integrals(const DevView& v, int c) {
  const InstParams& ip = v.inst[v.cell_inst[c]];
  const int nl = v.nl;
  const double H = v.cell_thck[c];
  const double* eq = v.eq3 + (size_t)c * 4 * nl;
  double* omk = v.cell_omk + (size_t)c * (nl + 1);
  double run[4] = {0.0, 0.0, 0.0, 0.0};
  omk[nl] = 0.0;
  for (int k = nl - 1; k >= 0; --k) {
    const double depth = 0.5 * (ip.sigma[k] + ip.sigma[k + 1]);
    const double dz = (ip.sigma[k + 1] - ip.sigma[k]) * H;
    double s = 0.0;
    for (int p = 0; p < 4; ++p) {
      run[p] = run[p] + depth / eq[(size_t)p * nl + k] * dz;
      s = s + run[p];
    }
    omk[k] = s / 4.0;
  }
  double om = 0.0;
  for (int k = 0; k < nl; ++k) om = om + 0.5 * (omk[k] + omk[k + 1]) * (ip.sigma[k + 1] - ip.sigma[k]);
  v.cell_om[c] = om;
}

// glissade_stagger with stagger_margin 1 over the ice-plus-land cells of
// column col (NW, NE, SW, SE) of a cell value val(cell) (zero for a cell
// the device does not hold: ice-free land).
template <typename F>
BP_HD double diva_stagger(const DevView& v, int col, F val) {
  const int nc = v.ncols;
  const uint8_t bits = v.col_ipl[col];
  const int order[4] = {2, 3, 0, 1};
  double s = 0.0;
  int n = 0;
  for (int o = 0; o < 4; ++o) {
    const int q = order[o];
    if (!((bits >> q) & 1)) continue;
    const int cell = v.col_cells[q * nc + col];
    s = s + (cell >= 0 ? val(cell) : 0.0);
    ++n;
  }
  return n > 0 ? s / (double)n : 0.0;
}

// beta_eff of column col (Goldberg 2011 eq. 40-41, :2750-2790): omega
// staggered to the vertex, beta_eff = beta / (1 + beta omega), or 1 /
// omega on a no-slip bed (0 where omega is 0).
BP_HD void diva_column_beta(const DevView& v, int col) {
  const InstParams& ip = v.inst[v.col_inst[col]];
  const double so = diva_stagger(v, col, [&](int cell) { return v.cell_om[cell]; });
  const double beta = v.col_beta[col];
  v.col_somega[col] = so;
  v.col_beff[col] = ip.which_babc == 6 ? (so > 0.0 ? 1.0 / so : 0.0) : beta / (1.0 + beta * so);
}

// After the linear solve (:3658-3696): the basal traction tau_b = beta_eff
// u_mean and compute_3d_velocity_diva (:5730-5830) for the mean velocity:
// u(bed) = u_mean - tau_b omega, u(k) = u(bed) + tau_b omega_k(k) with
// omega_k staggered level by level.
BP_HD void diva_column_velocity(const DevView& v, int col) {
  const int nl = v.nl;
  const double2 um = v.x[v.col_node[col]];
  const double be = v.col_beff[col], so = v.col_somega[col];
  double2 bt;
  bt.x = be * um.x;
  bt.y = be * um.y;
  v.col_bt[col] = bt;
  double2* out = v.x3 + (size_t)col * (nl + 1);
  double2 ub;
  ub.x = um.x - bt.x * so;
  ub.y = um.y - bt.y * so;
  out[nl] = ub;
  for (int k = 0; k < nl; ++k) {
    const double sk = diva_stagger(v, col, [&](int cell) { return v.cell_omk[(size_t)cell * (nl + 1) + k]; });
    double2 u;
    u.x = ub.x + bt.x * sk;
    u.y = ub.y + bt.y * sk;
    out[k] = u;
  }
}

// calcbeta (glissade_basal_traction.F90:67-598) at one vertex for the
// velocity-dependent laws, from the basal velocity (u, v) in m/a: the
// speed with its 0.01 m/a floor (:181) and optional cap (:187-189), the law
// (:207-264 pseudo-plastic, :266-277 yield stress, :357-363 power law,
// :365-382 power law with N, :384-424 Coulomb friction, :426-470
// Coulomb/power law after Schoof, :472-509 after Tsai), the grounded
// fraction (:540) and the grounded minimum (:560-566).  fg = f_ground; c1,
// c2 = the vertex's products formed before the speed enters (see
// SlideParams); the operations keep the reference's order.
BP_HD double slide_beta(const SlideParams& sp, double fg, double c1, double c2, double u,
                        double v) {
  const double smallnum = 1.0e-2;
  const double s0 = sqrt(u * u + v * v + smallnum * smallnum);
  double speed = s0;
  if (sp.umax > 0.0 && sp.umax < speed) speed = sp.umax;
  double beta = 0.0;
  switch (sp.law) {
    case 2:  // tau_y / |u|, from the uncapped speed
      beta = c1 / s0;
      break;
    case 3:  // tan(phi) N / (u0^q speed^(1-q))
      beta = c1 / (sp.k * pow(speed, sp.e1));
      break;
    case 9:  // C speed^(1/m - 1)
      beta = sp.c * pow(speed, sp.e2);
      break;
    case 10:  // c Cs N speed^(1/n - 1) (speed + N^n lambda)^(-1/n), at most 1e8
      beta = c1 * pow(speed, sp.e1) * pow(speed + c2, sp.e2);
      if (beta > 1.0e8) beta = 1.0e8;
      break;
    case 11: {  // C c N / (C^m speed + (c N)^m)^(1/m) speed^(1/m - 1), at most 1e8
      const double den = pow(sp.k * speed + c2, sp.e1);
      beta = (c1 / den) * pow(speed, sp.e2);
      if (beta > 1.0e8) beta = 1.0e8;
      break;
    }
    case 12: {  // min(c N, C speed^(1/m)) / speed
      const double tp = sp.c * pow(speed, sp.e1);
      beta = (c1 <= tp ? c1 : tp) / speed;
      break;
    }
    case 13:  // k^(-1/p) N^(q/p) speed^(1/p - 1)
      beta = c1 * pow(speed, sp.e1);
      break;
    default:
      break;
  }
  beta = beta * fg;
  if (fg > 0.0 && beta < sp.bmin) beta = sp.bmin;
  return beta;
}

// basal_sliding_bc (:8125-8381), bed layer only, diagonal blocks only.
template <int B>
BP_HD void row_basal(const DevView& v, const RefTables& T, int col, int k,
                     double* acc) {
  if (B != 0 && B != 3) return;
  if (k != v.nz - 1) return;
  const InstParams& ip = v.inst[v.col_inst[col]];
  // HO_BABC_NO_SLIP: no basal term, except for DIVA (beta_eff = 1/omega)
  if (ip.which_babc == 6 && !v.diva) return;
  if (ip.which_assemble_beta == 1) {  // HO_ASSEMBLE_BETA_LOCAL
    acc[13] += ip.dx * ip.dy / kVol0 * (v.diva ? v.col_beff[col] : v.col_beta[col]);
    return;
  }
  // standard: 2x2 face quadrature of beta * phi_r * phi_c on each bed face;
  // in-plane entries (kA = 0, stencil 9..17) gathered in a side array so
  // that acc keeps compile-time indices
  const int nc = v.ncols;
  const int nr_of_q[4] = {2, 3, 1, 0};  // 2-D node of this vertex in cells q = 0..3
  double bacc[9];
  for (int t = 0; t < 9; ++t) bacc[t] = 0.0;
  for (int qc = 0; qc < 4; ++qc) {
    const int cell = v.col_cells[qc * nc + col];
    if (cell < 0) continue;
    const int nr = nr_of_q[qc];
    const int ic = v.cell_ij[cell], jc = v.cell_ij[v.ncells + cell];
    const double xs[4] = {ip.dx * (ic - 1), ip.dx * ic, ip.dx * ic, ip.dx * (ic - 1)};
    const double ys[4] = {ip.dy * (jc - 1), ip.dy * (jc - 1), ip.dy * jc, ip.dy * jc};
    double b[4];
    for (int q = 0; q < 4; ++q) b[q] = v.cell_beta[q * v.ncells + cell];
    for (int p = 0; p < 4; ++p) {
      double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
      for (int n = 0; n < 4; ++n) {
        J11 += T.dxr2[p][n] * xs[n]; J12 += T.dxr2[p][n] * ys[n];
        J21 += T.dyr2[p][n] * xs[n]; J22 += T.dyr2[p][n] * ys[n];
      }
      const double detJ = J11 * J22 - J12 * J21;
      double bq = 0.0;
      for (int n = 0; n < 4; ++n) bq += T.phi2[p][n] * b[n];
      for (int ncn = 0; ncn < 4; ++ncn) {
        const double kv = bq * 1.0 * detJ / kVol0 * T.phi2[p][nr] * T.phi2[p][ncn];
        bacc[(node_di(ncn) - node_di(nr) + 1) + 3 * (node_dj(ncn) - node_dj(nr) + 1)] += kv;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 9; ++t) acc[9 + t] += bacc[t];
}

// dirichlet_boundary_conditions_3d (:8385-8578) restated row-locally: the
// row of node (col,k) is replaced when its own component is prescribed,
// and its entries toward prescribed neighbours are moved to the right-hand
// side.  Returns the sum moved to b (to be subtracted).
template <int B>
BP_HD double row_dirichlet(const DevView& v, int col, int k, double* acc) {
  const int nz = v.nz, nc = v.ncols;
  const uint8_t me = v.dmask[node_of(v, col, k)];
  const bool ur = me & 1, vr = me & 2;
  const bool row_presc = (B <= 1) ? ur : vr;
  double adj = 0.0;
  if (!row_presc && !v.any_dirichlet) return 0.0;
#pragma unroll
  for (int m = 0; m < 27; ++m) {
    const int iA = m % 3 - 1, jA = (m / 3) % 3 - 1, kA = m / 9 - 1;
    const bool diag = (m == 13);
    const int kn = k + kA;
    const int cn = v.col_nbr[((jA + 1) * 3 + (iA + 1)) * nc + col];
    const bool inb = (kn >= 0 && kn < nz && cn >= 0);
    if (row_presc) {
      if (inb || diag) acc[m] = (diag && (B == 0 || B == 3)) ? 1.0 : 0.0;
      continue;
    }
    if (!inb) continue;
    const size_t nn = node_of(v, cn, kn);
    const uint8_t pm = v.dmask[nn];
    if (diag) {
      // the reference zeroes the u-v coupling at a node whose other
      // component is prescribed, without moving it to the rhs
      if (B == 1 && vr) acc[m] = 0.0;
      if (B == 2 && ur) acc[m] = 0.0;
      continue;
    }
    const bool col_u = (B == 0 || B == 2);  // this block multiplies u of the neighbour
    const bool pres = col_u ? (pm & 1) : (pm & 2);
    if (pres) {
      const double2 xp = v.x[nn];
      adj += acc[m] * (col_u ? xp.x : xp.y);
      acc[m] = 0.0;
    }
  }
  return adj;
}

// ---------------------------------------------------------------------
// Structured 27-point block matvec, one row pair (u,v) of node (col,k):
// matvec_multiply_structured_3d (glissade_velo_higher_pcg.F90:2533-2647),
// same kA/jA/iA summation order.  SRC returns the source vector at a node.
// ---------------------------------------------------------------------
template <typename Mat, typename Src>
BP_HD double2 matvec_row(const DevView& v, const Mat* A, int col, int k, size_t n,
                         const Src& src) {
  const int nz = v.nz, nc = v.ncols;
  const size_t np = (size_t)v.npad;
  int cn[9];  // the neighbours' nodes at level 0
#pragma unroll
  for (int q = 0; q < 9; ++q) cn[q] = v.col_nbn[q * nc + col];
  double yu = 0.0, yv = 0.0;
#pragma unroll
  for (int kA = -1; kA <= 1; ++kA) {
    const int kn = k + kA;
    if (kn < 0 || kn >= nz) continue;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      if (cn[q] < 0) continue;
      const int m = (kA + 1) * 9 + q;
      const Mat au = BP_LD_STREAM(A + (size_t)m * np + n);
      const Mat av = BP_LD_STREAM(A + (size_t)(27 + m) * np + n);
      const double2 s = src((size_t)cn[q] + ((size_t)kn << v.lsh));
      yu += (double)au.x * s.x + (double)au.y * s.y;
      yv += (double)av.x * s.x + (double)av.y * s.y;
    }
  }
  return double2{yu, yv};
}

// ---------------------------------------------------------------------
// Symmetric storage.  Only stencil offsets m = 13..26 (the diagonal and the
// neighbours that come after the node in (kA, jA, iA) order) are stored per
// node; the entry toward an earlier neighbour P is the transpose of P's
// stored entry toward this node: Auu_m(R) = Auu_{26-m}(P),
// Auv_m(R) = Avu_{26-m}(P), Avu_m(R) = Auv_{26-m}(P), Avv_m(R) = Avv_{26-m}(P).
// Summed neighbour column by column (jA, iA outer, kA inner).
// ---------------------------------------------------------------------
BP_HD double diag_u(const DevView& v, size_t n) {
  return v.sym ? v.A[n].x : v.A[(size_t)13 * v.npad + n].x;
}
BP_HD double diag_v(const DevView& v, size_t n) {
  return v.sym ? v.A[(size_t)14 * v.npad + n].y : v.A[(size_t)(27 + 13) * v.npad + n].y;
}

template <typename View, typename Src>
BP_HD double2 matvec_row_sym(const View& v, const double2* A, int col, int k, size_t n,
                             const Src& src) {
  const int nz = v.nz, nc = v.ncols;
  const size_t np = (size_t)v.npad;
  double yu = 0.0, yv = 0.0;
  // neighbour columns outer (one node base serves three levels), as the FP32 body
#pragma unroll 3
  for (int q = 0; q < 9; ++q) {
    const int cq = v.col_nbn[q * nc + col];  // the neighbour column's node at level 0
#pragma unroll
    for (int kA = -1; kA <= 1; ++kA) {
      const int m = (kA + 1) * 9 + q, kn = k + kA;
      const bool ok = kn >= 0 && kn < nz && cq >= 0;
      const size_t p = ok ? (size_t)cq + ((size_t)kn << v.lsh) : n;  // in-bounds stand-in when absent
      double2 s = src(p);
      if (!ok) s = double2{0.0, 0.0};
      if (m >= 13) {
        const double2 a0 = BP_LD_RO(A + (size_t)(m - 13) * np + n);
        const double2 a1 = BP_LD_RO(A + (size_t)(14 + m - 13) * np + n);
        yu += a0.x * s.x + a0.y * s.y;
        yv += a1.x * s.x + a1.y * s.y;
      } else {
        const double2 b0 = BP_LD_RO(A + (size_t)(13 - m) * np + p);
        const double2 b1 = BP_LD_RO(A + (size_t)(14 + 13 - m) * np + p);
        yu += b0.x * s.x + b1.x * s.y;
        yv += b0.y * s.x + b1.y * s.y;
      }
    }
  }
  return double2{yu, yv};
}

// SIA column preconditioner (which_ho_precond = 2): z = M^-1 r with M the
// vertical tridiagonal of the uu and vv blocks, offsets m = 4, 13, 22
// (setup_preconditioner_3d, glissade_velo_higher_pcg.F90:2242-2252).
// Coefficients of node n (level k) in row h (0 u, 1 v); half storage reads
// the entry toward k-1 from the row below's entry toward k+1 (the uu and vv
// blocks are their own transposes).
BP_HD void sia_coefs(const DevView& v, size_t n, int k, int h, double* sub, double* dg, double* sup) {
  const size_t np = (size_t)v.npad;
  if (v.sym) {
    const double2 d = v.A[(size_t)(h * 14) * np + n];
    *dg = h ? d.y : d.x;
    if (k < v.nz - 1) {
      const double2 u = v.A[(size_t)(h * 14 + 9) * np + n];
      *sup = h ? u.y : u.x;
    } else {
      *sup = 0.0;
    }
    if (k > 0) {
      const double2 l = v.A[(size_t)(h * 14 + 9) * np + n - v.W];  // the node at k-1
      *sub = h ? l.y : l.x;
    } else {
      *sub = 0.0;
    }
  } else {
    const double2 d = v.A[(size_t)(h * 27 + 13) * np + n];
    *dg = h ? d.y : d.x;
    const double2 u = v.A[(size_t)(h * 27 + 22) * np + n];
    *sup = k < v.nz - 1 ? (h ? u.y : u.x) : 0.0;
    const double2 l = v.A[(size_t)(h * 27 + 4) * np + n];
    *sub = k > 0 ? (h ? l.y : l.x) : 0.0;
  }
}

// easy_sia_solver / tridiag_solver (pcg:2759-2904) in two halves.  The
// Thomas algorithm's forward elimination depends on the matrix only: per
// level k its pivot beta_k (beta_0 = d_0, beta_k = d_k - a_k gamma_k) and
// multiplier gamma_k = c_{k-1} / beta_{k-1} (gamma_0 = 0), with a, d, c the
// sub-, main and super-diagonal.  sia_factor_column forms them once per
// linear solve into v.sia_f [3][npad] ((a, beta, gamma) per node, u and v
// components); every preconditioner application then runs the two sweeps
// (sia_solve) in the reference's order and operations, so the result is
// that of the reference's solver bitwise.
BP_HD void sia_factor_column(const DevView& v, int col, int h) {
  const size_t np = (size_t)v.npad;
  double beta = 0.0, sup_prev = 0.0;
  for (int k = 0; k < v.nz; ++k) {
    const size_t n = node_of(v, col, k);
    double sub, dg, sup;
    sia_coefs(v, n, k, h, &sub, &dg, &sup);
    double gam = 0.0;
    if (k == 0) {
      beta = dg;
    } else {
      gam = sup_prev / beta;
      beta = dg - sub * gam;
    }
    sup_prev = sup;
    double* f = reinterpret_cast<double*>(v.sia_f);
    f[(n) * 2 + h] = sub;
    f[(np + n) * 2 + h] = beta;
    f[(2 * np + n) * 2 + h] = gam;
  }
}

// The two sweeps for one column and component: s holds r on entry and z on
// exit, level k at s[k * stride]; fac(k) gives level k's factors (sub-
// diagonal a, pivot beta, multiplier gamma).
struct SiaFac {
  double a, beta, gam;
};

template <typename Fac>
BP_HD void sia_sweeps(int nz, const Fac& fac, double* s, int stride) {
  s[0] = s[0] / fac(0).beta;
  for (int k = 1; k < nz; ++k) {
    const SiaFac f = fac(k);
    s[k * stride] = (s[k * stride] - f.a * s[(k - 1) * stride]) / f.beta;
  }
  for (int k = nz - 2; k >= 0; --k) s[k * stride] = s[k * stride] - fac(k + 1).gam * s[(k + 1) * stride];
}

// The sweeps with the factors read from v.sia_f: node(k) is the column's
// node at level k, h the component.
template <typename NodeOf>
BP_HD void sia_solve(const DevView& v, int nz, int h, NodeOf node, double* s, int stride) {
  const size_t np = (size_t)v.npad;
  const double* f = reinterpret_cast<const double*>(v.sia_f);
  sia_sweeps(
      nz,
      [&](int k) {
        const size_t n = node(k);
        return SiaFac{f[n * 2 + h], f[(np + n) * 2 + h], f[(2 * np + n) * 2 + h]};
      },
      s, stride);
}

// FP32 copy of row n of the symmetric matrix for the mixed-precision
// Krylov matvecs.  Rounding each entry to FP32 perturbs the row sums, and
// with them the operator on smooth fields (the translation modes are
// nearly in its null space), by about eps32 times the unpreconditioned
// condition number, which stalls the Krylov iteration.  The FP64 diagonal
// block therefore takes up the rounding of every off-diagonal entry of its
// row (all 27 offsets, the lower ones read from the neighbours' stored
// blocks as the matvec reads them), so that the FP32 operator keeps the
// FP64 row sums exactly.
BP_HD double rd_err32(double a) { return a - (double)(float)a; }

BP_HD void make_a32_row(const DevView& v, int col, int k, size_t n) {
  const size_t np = (size_t)v.npad;
  const int nz = v.nz, nc = v.ncols;
  for (int mm = 0; mm < 14; ++mm) {
    const double2 a = v.A[(size_t)mm * np + n], b = v.A[(size_t)(14 + mm) * np + n];
    v.A32[(size_t)mm * np + n] = float4{(float)a.x, (float)a.y, (float)b.x, (float)b.y};
  }
  int cn[9];  // the neighbours' nodes at level 0
  for (int q = 0; q < 9; ++q) cn[q] = v.col_nbn[q * nc + col];
  double euu = 0.0, euv = 0.0, evu = 0.0, evv = 0.0;
  for (int m = 0; m < 27; ++m) {
    if (m == 13) continue;
    const int kn = k + m / 9 - 1, q = m % 9;
    if (kn < 0 || kn >= nz || cn[q] < 0) continue;
    if (m > 13) {
      const double2 a = v.A[(size_t)(m - 13) * np + n], b = v.A[(size_t)(m + 1) * np + n];
      euu += rd_err32(a.x);
      euv += rd_err32(a.y);
      evu += rd_err32(b.x);
      evv += rd_err32(b.y);
    } else {
      const size_t p = (size_t)cn[q] + ((size_t)kn << v.lsh);
      const double2 b0 = v.A[(size_t)(13 - m) * np + p], b1 = v.A[(size_t)(27 - m) * np + p];
      euu += rd_err32(b0.x);
      euv += rd_err32(b1.x);
      evu += rd_err32(b0.y);
      evv += rd_err32(b1.y);
    }
  }
  const double2 d0 = v.A[n], d1 = v.A[(size_t)14 * np + n];
  v.A32d[n] = double2{d0.x + euu, d0.y + euv};
  v.A32d[np + n] = double2{d1.x + evu, d1.y + evv};
}

// FP32 symmetric storage, (uu, uv, vu, vv) packed per offset, with the
// row-sum compensated diagonal block in FP64; FP64 sums.  The neighbour
// columns are the outer loop, unrolled by three: each column's node base is
// read once and serves its three levels, so few bases are live at a time
// and six to eight CTAs of the tile fit an SM (26% faster than holding all
// nine bases with the levels outer, on a 1.9M-node batch).
template <typename Src>
BP_HD double2 matvec_row_sym32(const DevView& v, const float4* A, int col, int k, size_t n,
                               const Src& src) {
  const int nz = v.nz, nc = v.ncols;
  const size_t np = (size_t)v.npad;
  double yu = 0.0, yv = 0.0;
#pragma unroll 3
  for (int q = 0; q < 9; ++q) {
    const int cq = v.col_nbn[q * nc + col];  // the neighbour column's node at level 0
#pragma unroll
    for (int kA = -1; kA <= 1; ++kA) {
      const int m = (kA + 1) * 9 + q, kn = k + kA;
      const bool ok = kn >= 0 && kn < nz && cq >= 0;
      const size_t p = ok ? (size_t)cq + ((size_t)kn << v.lsh) : n;  // in-bounds stand-in when absent
      double2 s = src(p);
      if (!ok) s = double2{0.0, 0.0};
      if (m == 13) {
        const double2 a0 = BP_LD_RO(v.A32d + n), a1 = BP_LD_RO(v.A32d + np + n);
        yu += a0.x * s.x + a0.y * s.y;
        yv += a1.x * s.x + a1.y * s.y;
      } else if (m > 13) {
        const float4 a = BP_LD_RO(A + (size_t)(m - 13) * np + n);
        yu += (double)a.x * s.x + (double)a.y * s.y;
        yv += (double)a.z * s.x + (double)a.w * s.y;
      } else {
        const float4 b = BP_LD_RO(A + (size_t)(13 - m) * np + p);
        yu += (double)b.x * s.x + (double)b.z * s.y;
        yv += (double)b.y * s.x + (double)b.w * s.y;
      }
    }
  }
  return double2{yu, yv};
}

}  // namespace bp
