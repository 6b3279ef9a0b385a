// bp_setup.cpp -- host-side mirror of the setup part of
// glissade_velo_higher_solve (libglissade/glissade_velo_higher.F90:987-2199),
// for callers that hold model fields instead of the boundary inputs.  It
// runs once per solve on O(cells) data; the Picard loop itself runs on the
// device (bp_solve).
#include <cmath>
#include <cstring>
#include <vector>

#include "bp_b200.h"
#include "bp_plan.h"

namespace {

// Fortran-order views with 1-based indices.
struct Cells {
  int nx, ny;
  size_t operator()(int i, int j) const { return (size_t)(j - 1) * nx + (i - 1); }
};
struct Verts {
  int nx, ny;  // cell counts; vertices are (nx-1) x (ny-1)
  size_t operator()(int i, int j) const { return (size_t)(j - 1) * (nx - 1) + (i - 1); }
};

template <typename T>
void halo_cells(int nx, int ny, int periodic, T* a) {
  Cells C{nx, ny};
  if (!periodic) {
    for (int j = 3; j <= ny - 2; ++j) a[C(1, j)] = a[C(2, j)] = a[C(nx - 1, j)] = a[C(nx, j)] = 0;
    for (int i = 1; i <= nx; ++i) a[C(i, 1)] = a[C(i, 2)] = a[C(i, ny - 1)] = a[C(i, ny)] = 0;
    return;
  }
  for (int j = 3; j <= ny - 2; ++j) {
    const T e1 = a[C(nx - 3, j)], e2 = a[C(nx - 2, j)], w1 = a[C(3, j)], w2 = a[C(4, j)];
    a[C(1, j)] = e1; a[C(2, j)] = e2; a[C(nx - 1, j)] = w1; a[C(nx, j)] = w2;
  }
  for (int i = 1; i <= nx; ++i) {
    const T n1 = a[C(i, ny - 3)], n2 = a[C(i, ny - 2)], s1 = a[C(i, 3)], s2 = a[C(i, 4)];
    a[C(i, 1)] = n1; a[C(i, 2)] = n2; a[C(i, ny - 1)] = s1; a[C(i, ny)] = s2;
  }
}

// MIN/MAX with a NaN operand return the other operand.
double ramp_factor(double thck, double thklim, double ramp) {
  return std::fmax(std::fmin(1.0, (thck - thklim) / ramp), 0.0);
}

}  // namespace

extern "C" int bp_setup(const bp_model* m, bp_setup_arrays* o, double* uvel,
                        double* vvel, bp_inputs* in) {
  if (!m || !o || !uvel || !vvel) return BP_ERR_ARGS;
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  if (m->nhalo != 2 || nx < 6 || ny < 6 || nz < 2 || nz > bp::kNzMax) return BP_ERR_ARGS;
  if (!m->thck || !m->usrf || !m->topg || !m->flwa) return BP_ERR_ARGS;
  // options this mirror restates: centred or upstream surface gradient
  // with the land, hybrid or marine margin rule; grounded fraction without the
  // grounding-line parameterisation, or all grounded (a caller with other
  // options computes bp_inputs itself)
  if (m->which_gradient < 0 || m->which_gradient > 2 || m->which_gradient_margin < 0 ||
      m->which_gradient_margin > 2 ||
      (m->which_ground != 0 && m->which_ground != 2) ||
      (m->which_assemble_taud != 0 && m->which_assemble_taud != 1) ||
      (m->which_assemble_beta != 0 && m->which_assemble_beta != 1))
    return BP_ERR_ARGS;
  // basal traction: constant, external or no slip here; the
  // velocity-dependent laws through m->sliding; the other calcbeta options
  // (BPMP, large, ISMIP-HOM C, the simple pattern) come in as beta_internal
  // of a caller-built bp_inputs
  if (!m->sliding && m->which_babc != 0 && m->which_babc != 5 && m->which_babc != 6) return BP_ERR_ARGS;
  if (m->sliding && (m->sliding->law != m->which_babc || !o->f_ground ||
                     (m->sliding->law == 10 && !o->flwa_basal_stag)))
    return BP_ERR_ARGS;
  // 3-D Blatter-Pattyn, or the shallow-shelf, L1L2 or DIVA 2-D solve
  if (m->approx_2d != 0 && m->approx_2d != 1 && m->approx_2d != 3 && m->approx_2d != 4) return BP_ERR_ARGS;
  if (m->approx_2d == 3 && (!o->dusrf_dx || !o->dusrf_dy)) return BP_ERR_ARGS;
  const bool diva = m->approx_2d == 4;
  if (diva && (!m->diva || !m->diva->uvel_2d || !m->diva->vvel_2d || !m->diva->btractx ||
               !m->diva->btracty || !o->ice_plus_land_mask))
    return BP_ERR_ARGS;
  const Cells C{nx, ny};
  const Verts V{nx, ny};
  const size_t ncell = (size_t)nx * ny, nvert = (size_t)(nx - 1) * (ny - 1), n3 = nvert * nz;

  // sigma levels: Glide default, glide_setup.F90:281-290
  std::vector<double> wbnd(nz + 1);
  for (int k = 0; k < nz; ++k) {
    const double lev = (double)k / (double)(nz - 1);
    o->sigma[k] = (1.0 - std::pow(lev + 1.0, -2.0)) / (1.0 - std::pow(2.0, -2.0));
  }
  wbnd[0] = 0.0;
  for (int k = 1; k < nz; ++k) wbnd[k] = (o->sigma[k - 1] + o->sigma[k]) / 2.0;
  wbnd[nz] = 1.0;

  // Dirichlet masks, :1270-1324
  std::memset(o->umask_dirichlet, 0, n3 * sizeof(int));
  std::memset(o->vmask_dirichlet, 0, n3 * sizeof(int));
  for (size_t v = 0; v < nvert; ++v) {
    // DIVA takes a no-slip bed through beta_eff = 1/omega (:1274-1278)
    const bool noslip = m->which_babc == 6 && !diva;
    const bool kin = m->kinbcmask && m->kinbcmask[v] == 1;
    for (int k = 0; k < nz; ++k)
      if (kin || (noslip && k == nz - 1)) {
        o->umask_dirichlet[v * nz + k] = 1;
        o->vmask_dirichlet[v * nz + k] = 1;
      }
    if (kin && diva) {  // a 2-D solve's Dirichlet column starts from its bed velocity (:1300-1303)
      m->diva->uvel_2d[v] = uvel[v * nz + nz - 1];
      m->diva->vvel_2d[v] = vvel[v * nz + nz - 1];
    }
  }

  // masks, glissade_masks.F90:55-457 (no sub-grid calving front)
  std::vector<int> ice(ncell), flt(ncell), ocean(ncell), land(ncell);
  for (size_t c = 0; c < ncell; ++c) {
    ice[c] = m->thck[c] > m->thklim;
    ocean[c] = m->topg[c] < m->eus && !ice[c];
    flt[c] = ice[c] && (m->topg[c] - m->eus < (-m->rhoi / m->rhoo) * m->thck[c]);
    land[c] = m->topg[c] >= m->eus;
  }
  halo_cells(nx, ny, m->periodic, ice.data());
  halo_cells(nx, ny, m->periodic, flt.data());
  const std::vector<int>& active_ice = ice;
  std::vector<int> ipl(ncell);
  for (size_t c = 0; c < ncell; ++c) ipl[c] = active_ice[c] || land[c];
  if (diva)
    for (size_t c = 0; c < ncell; ++c) o->ice_plus_land_mask[c] = ipl[c];

  // glissade_stagger with stagger_margin = 1, glissade_grid_operators.F90:60-148
  auto stagger = [&](const double* var, double* out) {
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        const int w[4] = {ipl[C(i, j + 1)], ipl[C(i + 1, j + 1)], ipl[C(i, j)], ipl[C(i + 1, j)]};
        const double s = w[0] * var[C(i, j + 1)] + w[1] * var[C(i + 1, j + 1)] +
                         w[2] * var[C(i, j)] + w[3] * var[C(i + 1, j)];
        const double n = (double)(w[0] + w[1] + w[2] + w[3]);
        out[V(i, j)] = n > 0.0 ? s / n : 0.0;
      }
  };
  stagger(m->thck, o->stagthck);
  stagger(m->usrf, o->stagusrf);

  // surface gradient on vertices (glissade_surface_elevation_gradient,
  // glissade_grid_operators.F90:734-1168): edge gradients by the margin
  // option, then centred, first- or second-order upstream vertex values
  std::vector<double> gx(ncell, 0.0), gy(ncell, 0.0), dsdx(nvert), dsdy(nvert);
  auto edge = [&](int ia, int ja, int ib, int jb, double d) -> double {
    // gradient from cell a to the next cell b along one axis
    const double sa = m->usrf[C(ia, ja)], sb = m->usrf[C(ib, jb)];
    if (m->which_gradient_margin == 0) return (sb - sa) / d;
    if (m->which_gradient_margin == 2)
      return (active_ice[C(ia, ja)] && active_ice[C(ib, jb)]) ? (sb - sa) / d : 0.0;
    const bool a_up = sa > sb;
    const size_t up = a_up ? C(ia, ja) : C(ib, jb), lo = a_up ? C(ib, jb) : C(ia, ja);
    const double sgn = a_up ? -1.0 : 1.0;
    const double f = land[up] ? ramp_factor(m->thck[up], m->thklim, m->thck_gradient_ramp) : 1.0;
    if (active_ice[up] && (active_ice[lo] || land[lo])) return f * sgn * (m->usrf[up] - m->usrf[lo]) / d;
    return 0.0;
  };
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx - 1; ++i) gx[C(i, j)] = edge(i, j, i + 1, j, m->dx);
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx; ++i) gy[C(i, j)] = edge(i, j, i, j + 1, m->dy);
  const double* sf = m->usrf;
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      double a = 0.0, b = 0.0;
      if (m->which_gradient == 0) {  // centred (:983-1026)
        a = 0.5 * (gx[C(i, j)] + gx[C(i, j + 1)]);
        b = 0.5 * (gy[C(i, j)] + gy[C(i + 1, j)]);
      } else if (m->which_gradient == 1) {  // the edge on the higher side (:1028-1058)
        a = (sf[C(i, j + 1)] + sf[C(i + 1, j + 1)] > sf[C(i, j)] + sf[C(i + 1, j)]) ? gx[C(i, j + 1)]
                                                                                    : gx[C(i, j)];
        b = (sf[C(i + 1, j)] + sf[C(i + 1, j + 1)] > sf[C(i, j)] + sf[C(i, j + 1)]) ? gy[C(i + 1, j)]
                                                                                    : gy[C(i, j)];
      } else if (i >= 2 && i <= nx - 2 && j >= 2 && j <= ny - 2) {  // two edges upstream (:1060-1093)
        const bool north = sf[C(i, j + 1)] + sf[C(i + 1, j + 1)] + sf[C(i, j + 2)] + sf[C(i + 1, j + 2)] >
                           sf[C(i, j)] + sf[C(i + 1, j)] + sf[C(i, j - 1)] + sf[C(i + 1, j - 1)];
        a = north ? 1.5 * gx[C(i, j + 1)] - 0.5 * gx[C(i, j + 2)] : 1.5 * gx[C(i, j)] - 0.5 * gx[C(i, j - 1)];
        const bool east = sf[C(i + 1, j)] + sf[C(i + 1, j + 1)] + sf[C(i + 2, j)] + sf[C(i + 2, j + 1)] >
                          sf[C(i, j)] + sf[C(i, j + 1)] + sf[C(i - 1, j)] + sf[C(i - 1, j + 1)];
        b = east ? 1.5 * gy[C(i + 1, j)] - 0.5 * gy[C(i + 2, j)] : 1.5 * gy[C(i, j)] - 0.5 * gy[C(i - 1, j)];
      }
      a = a > 0.0 ? std::fmin(a, m->max_slope) : std::fmax(a, -m->max_slope);
      b = b > 0.0 ? std::fmin(b, m->max_slope) : std::fmax(b, -m->max_slope);
      dsdx[V(i, j)] = a;
      dsdy[V(i, j)] = b;
    }
  bp::halo_stag(nx, ny, 1, m->periodic, dsdx.data());
  bp::halo_stag(nx, ny, 1, m->periodic, dsdy.data());
  if (m->approx_2d == 3) {  // the L1L2 viscosity and reconstruction read it
    std::memcpy(o->dusrf_dx, dsdx.data(), nvert * sizeof(double));
    std::memcpy(o->dusrf_dy, dsdy.data(), nvert * sizeof(double));
  }

  // get_vertex_geometry, :4163-4313
  std::memset(o->active_cell, 0, ncell * sizeof(int));
  std::memset(o->active_vertex, 0, nvert * sizeof(int));
  for (int j = 3; j <= ny - 1; ++j)
    for (int i = 3; i <= nx - 1; ++i)
      if (active_ice[C(i, j)]) {
        o->active_cell[C(i, j)] = 1;
        o->active_vertex[V(i - 1, j - 1)] = o->active_vertex[V(i, j - 1)] = 1;
        o->active_vertex[V(i - 1, j)] = o->active_vertex[V(i, j)] = 1;
      }
  const bp::OwnedRange R = bp::owned_range(nx, ny, m->periodic);
  for (int j = R.jlo; j <= R.jhi; ++j)
    for (int i = R.ilo; i <= R.ihi; ++i)
      if (!o->active_vertex[V(i, j)]) {
        for (int k = 0; k < nz; ++k) uvel[V(i, j) * nz + k] = vvel[V(i, j) * nz + k] = 0.0;
        if (diva) m->diva->uvel_2d[V(i, j)] = m->diva->vvel_2d[V(i, j)] = 0.0;
      }

  // flwafact = 0.5 A^(-1/n), :1919-1939
  std::memset(o->flwafact, 0, (size_t)(nz - 1) * ncell * sizeof(double));
  for (int j = 3; j <= ny - 1; ++j)
    for (int i = 3; i <= nx - 1; ++i)
      for (int k = 0; k < nz - 1; ++k) {
        const double a = m->flwa[C(i, j) * (nz - 1) + k];
        if (a > 0.0) o->flwafact[C(i, j) * (nz - 1) + k] = 0.5 * std::pow(a, -1.0 / 3.0);
      }

  // load vector: gravity (:4317-4532, local assembly) and lateral
  // ocean-face pressure (:4536-4950)
  std::memset(o->loadu, 0, n3 * sizeof(double));
  std::memset(o->loadv, 0, n3 * sizeof(double));
  const double vol0 = bp::kVol0, rg = m->rhoi * m->grav;
  if (m->which_assemble_taud == 1) {
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        if (!o->active_vertex[V(i, j)]) continue;
        for (int k = 0; k < nz; ++k) {
          const double dz = o->stagthck[V(i, j)] * (wbnd[k + 1] - wbnd[k]);
          o->loadu[V(i, j) * nz + k] -= rg * m->dx * m->dy * dz / vol0 * dsdx[V(i, j)];
          o->loadv[V(i, j) * nz + k] -= rg * m->dx * m->dy * dz / vol0 * dsdy[V(i, j)];
        }
      }
  } else {
    // standard assembly (:4436-4528): rho g ds/dx integrated against every
    // basis function over the elements of the active cells, 2x2x2 Gauss
    // points, with the surface gradient interpolated to each point
    const double r = 1.0 / std::sqrt(3.0);
    const double sgx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const double sgy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const double sgz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    double phi[8][8], dxi[8][8], deta[8][8], dzeta[8][8];  // [p][n]
    for (int q = 0; q < 8; ++q) {
      const double xq = sgx[q] * r, yq = sgy[q] * r, zq = sgz[q] * r;
      for (int n = 0; n < 8; ++n) {
        phi[q][n] = (1.0 + sgx[n] * xq) * (1.0 + sgy[n] * yq) * (1.0 + sgz[n] * zq) / 8.0;
        dxi[q][n] = sgx[n] * (1.0 + sgy[n] * yq) * (1.0 + sgz[n] * zq) / 8.0;
        deta[q][n] = sgy[n] * (1.0 + sgx[n] * xq) * (1.0 + sgz[n] * zq) / 8.0;
        dzeta[q][n] = sgz[n] * (1.0 + sgx[n] * xq) * (1.0 + sgy[n] * yq) / 8.0;
      }
    }
    for (int j = 3; j <= ny - 1; ++j)
      for (int i = 3; i <= nx - 1; ++i) {
        if (!o->active_cell[C(i, j)]) continue;
        for (int k = 0; k < nz - 1; ++k) {
          // nodes SW, SE, NE, NW of the lower face (level k+1), then the upper face (level k)
          int vi[8], vj[8], lv[8];
          double x[8], y[8], z[8], gx8[8], gy8[8];
          for (int n = 0; n < 8; ++n) {
            const int c = n & 3;
            vi[n] = (c == 1 || c == 2) ? i : i - 1;
            vj[n] = c >= 2 ? j : j - 1;
            lv[n] = n < 4 ? k + 1 : k;
            const size_t w = V(vi[n], vj[n]);
            x[n] = m->dx * vi[n];
            y[n] = m->dy * vj[n];
            z[n] = o->stagusrf[w] - o->sigma[lv[n]] * o->stagthck[w];
            gx8[n] = dsdx[w];
            gy8[n] = dsdy[w];
          }
          for (int q = 0; q < 8; ++q) {
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int n = 0; n < 8; ++n) {
              J[0][0] = J[0][0] + dxi[q][n] * x[n];
              J[0][1] = J[0][1] + dxi[q][n] * y[n];
              J[0][2] = J[0][2] + dxi[q][n] * z[n];
              J[1][0] = J[1][0] + deta[q][n] * x[n];
              J[1][1] = J[1][1] + deta[q][n] * y[n];
              J[1][2] = J[1][2] + deta[q][n] * z[n];
              J[2][0] = J[2][0] + dzeta[q][n] * x[n];
              J[2][1] = J[2][1] + dzeta[q][n] * y[n];
              J[2][2] = J[2][2] + dzeta[q][n] * z[n];
            }
            // detJ by cofactor expansion along the first row (:6439-6464)
            const double c0 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
            const double c1 = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]);
            const double c2 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
            const double detJ = J[0][0] * c0 + J[0][1] * c1 + J[0][2] * c2;
            double gxq = 0.0, gyq = 0.0;
            for (int n = 0; n < 8; ++n) {
              gxq = gxq + phi[q][n] * gx8[n];
              gyq = gyq + phi[q][n] * gy8[n];
            }
            for (int n = 0; n < 8; ++n) {
              const size_t t = V(vi[n], vj[n]) * nz + lv[n];
              o->loadu[t] = o->loadu[t] - rg * 1.0 * detJ / vol0 * gxq * phi[q][n];
              o->loadv[t] = o->loadv[t] - rg * 1.0 * detJ / vol0 * gyq * phi[q][n];
            }
          }
        }
      }
  }
  const double r3 = 1.0 / std::sqrt(3.0);
  const double qx[4] = {-r3, r3, r3, -r3}, qy[4] = {-r3, -r3, r3, r3};
  auto face = [&](int dir, int ic, int jc) {
    // dir: 0 west, 1 east, 2 south, 3 north; nodes along the face
    int a[2][2];
    if (dir == 0) { a[0][0] = ic - 1; a[0][1] = jc; a[1][0] = ic - 1; a[1][1] = jc - 1; }
    else if (dir == 1) { a[0][0] = ic; a[0][1] = jc - 1; a[1][0] = ic; a[1][1] = jc; }
    else if (dir == 2) { a[0][0] = ic - 1; a[0][1] = jc - 1; a[1][0] = ic; a[1][1] = jc - 1; }
    else { a[0][0] = ic; a[0][1] = jc; a[1][0] = ic - 1; a[1][1] = jc; }
    const double h0 = o->stagthck[V(a[0][0], a[0][1])], h1 = o->stagthck[V(a[1][0], a[1][1])];
    const double s0 = o->stagusrf[V(a[0][0], a[0][1])], s1 = o->stagusrf[V(a[1][0], a[1][1])];
    const double c0 = dir <= 1 ? m->dy * a[0][1] : m->dx * a[0][0];
    const double c1 = dir <= 1 ? m->dy * a[1][1] : m->dx * a[1][0];
    const double xs[4] = {c0, c1, c1, c0};
    const double hs[4] = {h0, h1, h1, h0}, ss[4] = {s0, s1, s1, s0};
    for (int k = 0; k < nz - 1; ++k) {
      const double ys[4] = {s0 - o->sigma[k + 1] * h0, s1 - o->sigma[k + 1] * h1,
                            s1 - o->sigma[k] * h1, s0 - o->sigma[k] * h0};
      const int lev[4] = {k + 1, k + 1, k, k};
      for (int p = 0; p < 4; ++p) {
        double phi[4], dxi[4], deta[4];
        for (int n = 0; n < 4; ++n) {
          const double sx = (n == 1 || n == 2) ? 1.0 : -1.0, sy = (n >= 2) ? 1.0 : -1.0;
          phi[n] = (1.0 + sx * qx[p]) * (1.0 + sy * qy[p]) / 4.0;
          dxi[n] = sx * (1.0 + sy * qy[p]) / 4.0;
          deta[n] = sy * (1.0 + sx * qx[p]) / 4.0;
        }
        double J11 = 0, J12 = 0, J21 = 0, J22 = 0, hq = 0, sq = 0;
        for (int n = 0; n < 4; ++n) {
          J11 += dxi[n] * xs[n]; J12 += dxi[n] * ys[n];
          J21 += deta[n] * xs[n]; J22 += deta[n] * ys[n];
          hq += phi[n] * hs[n]; sq += phi[n] * ss[n];
        }
        const double detJ = std::fabs(J11 * J22 - J12 * J21);
        const double t = 1.0 - std::fmin(sq / hq, 1.0);
        const double pav = 0.5 * rg * hq - 0.5 * m->rhoo * m->grav * hq * (t * t);
        for (int n = 0; n < 4; ++n) {
          const int vi = (n == 0 || n == 3) ? a[0][0] : a[1][0];
          const int vj = (n == 0 || n == 3) ? a[0][1] : a[1][1];
          const double f = pav * detJ / vol0 * phi[n];
          double* L = (dir <= 1) ? o->loadu : o->loadv;
          const double sgn = (dir == 0 || dir == 2) ? -1.0 : 1.0;
          L[V(vi, vj) * nz + lev[n]] += sgn * f;
        }
      }
    }
  };
  for (int j = 3; j <= ny - 1; ++j)
    for (int i = 3; i <= nx - 1; ++i) {
      if (!o->active_cell[C(i, j)]) continue;
      if (ocean[C(i - 1, j)]) face(0, i, j);
      if (ocean[C(i + 1, j)]) face(1, i, j);
      if (ocean[C(i, j - 1)]) face(2, i, j);
      if (ocean[C(i, j + 1)]) face(3, i, j);
    }

  // grounded fraction (glissade_grounding_line.F90:55-178, NO_GLP; the
  // reference tests land_mask(i+1,j+1) twice and never land_mask(i+1,j))
  // and calcbeta (glissade_basal_traction.F90:67-598, constant/external)
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const size_t c00 = C(i, j), c10 = C(i + 1, j), c01 = C(i, j + 1), c11 = C(i + 1, j + 1);
      const bool vmask = ice[c01] || ice[c11] || ice[c00] || ice[c10] || land[c01] || land[c11] ||
                         land[c00] || land[c11];
      double fg = 0.0;
      if (vmask) {
        if (m->which_ground == 2) fg = 1.0;
        else {
          auto cg = [&](size_t c) { return (ice[c] && !flt[c]) || land[c]; };
          fg = (cg(c01) || cg(c11) || cg(c00) || cg(c10)) ? 1.0 : 0.0;
        }
      }
      double b = m->which_babc == 0 ? m->beta_const
               : (m->beta_external ? m->beta_external[V(i, j)] : 0.0);
      if (m->which_babc != 0 && m->which_babc != 5) b = 0.0;
      b = b * fg;
      if (fg > 0.0 && b < m->beta_grounded_min) b = m->beta_grounded_min;
      if (!(b >= 0.0)) return BP_ERR_BAD_BETA;
      o->beta_internal[V(i, j)] = b;
      if (m->sliding) o->f_ground[V(i, j)] = fg;
    }
  bp::halo_stag(nx, ny, 1, m->periodic, o->beta_internal);

  // velocity-dependent sliding law: the solve evaluates it every Picard
  // iteration from f_ground and, for Coulomb friction, the basal layer's
  // flow factor staggered over cells with thck > 0
  // (glissade_basal_traction.F90:393-398, glissade_stagger margin 1)
  if (m->sliding) {
    if (m->sliding->law == 10) {
      for (int j = 1; j <= ny - 1; ++j)
        for (int i = 1; i <= nx - 1; ++i) {
          const size_t cc[4] = {C(i, j + 1), C(i + 1, j + 1), C(i, j), C(i + 1, j)};
          double sumvar = 0.0;
          int summask = 0;
          for (int q = 0; q < 4; ++q) {
            const int w = m->thck[cc[q]] > 0.0 ? 1 : 0;
            const double term = (double)w * m->flwa[cc[q] * (nz - 1) + (nz - 2)];
            sumvar = q == 0 ? term : sumvar + term;
            summask += w;
          }
          o->flwa_basal_stag[V(i, j)] = summask > 0 ? sumvar / (double)summask : 0.0;
        }
    }
    o->sliding = *m->sliding;
    o->sliding.f_ground = o->f_ground;
    o->sliding.topg = m->topg;
    o->sliding.eus = m->eus;
    o->sliding.beta_grounded_min = m->beta_grounded_min;
    if (m->sliding->law == 10) o->sliding.flwa_basal_stag = o->flwa_basal_stag;
  }

  if (in) {
    std::memset(in, 0, sizeof(*in));
    in->nx = nx; in->ny = ny; in->nz = nz; in->nhalo = 2; in->periodic = m->periodic;
    in->dx = m->dx; in->dy = m->dy;
    in->sigma = o->sigma; in->stagusrf = o->stagusrf; in->stagthck = o->stagthck;
    in->beta_internal = o->beta_internal; in->flwafact = o->flwafact;
    in->active_cell = o->active_cell; in->active_vertex = o->active_vertex;
    in->loadu = o->loadu; in->loadv = o->loadv;
    in->umask_dirichlet = o->umask_dirichlet; in->vmask_dirichlet = o->vmask_dirichlet;
    in->which_babc = m->which_babc; in->which_efvs = m->which_efvs;
    in->efvs_constant = m->efvs_constant; in->which_assemble_beta = m->which_assemble_beta;
    in->which_resid = m->which_resid;
    in->pcg_variant = m->which_sparse == 3 ? 3 : 2;
    in->which_precond = m->which_precond;
    in->maxiter_nonlinear = m->maxiter_nonlinear;
    in->pcg_maxiters = m->pcg_maxiters; in->pcg_ncheck = m->pcg_ncheck; in->pcg_tol = m->pcg_tol;
    in->precision = m->precision; in->inner_tol = m->inner_tol;
    in->sliding = m->sliding ? &o->sliding : nullptr;
    in->approx_2d = m->approx_2d;
    if (m->approx_2d == 3) {
      o->l1l2.thck = m->thck;
      o->l1l2.flwa = m->flwa;
      o->l1l2.dusrf_dx = o->dusrf_dx;
      o->l1l2.dusrf_dy = o->dusrf_dy;
      o->l1l2.rhoi = m->rhoi;
      o->l1l2.grav = m->grav;
      in->l1l2 = &o->l1l2;
    }
    if (diva) {
      o->diva = *m->diva;
      o->diva.thck = m->thck;
      o->diva.ice_plus_land_mask = o->ice_plus_land_mask;
      in->diva = &o->diva;
    }
  }
  return BP_OK;
}

extern "C" int bp_velo_higher_solve(bp_ctx* ctx, const bp_model* m, double* uvel,
                                    double* vvel, double* efvs, bp_stats* stats) {
  if (!ctx || !m) return BP_ERR_ARGS;
  const size_t ncell = (size_t)m->nx * m->ny, nvert = (size_t)(m->nx - 1) * (m->ny - 1);
  const size_t n3 = nvert * m->nz;
  std::vector<double> sigma(m->nz), su(nvert), sh(nvert), beta(nvert),
      fl((size_t)(m->nz - 1) * ncell), lu(n3), lv(n3);
  std::vector<int> ac(ncell), av(nvert), um(n3), vm(n3);
  std::vector<double> fg(m->sliding ? nvert : 0), fbs(m->sliding ? nvert : 0);
  std::vector<double> gx(m->approx_2d == 3 ? nvert : 0), gy(m->approx_2d == 3 ? nvert : 0);
  std::vector<int> iplm(m->approx_2d == 4 ? ncell : 0);
  bp_setup_arrays o{};
  o.sigma = sigma.data(); o.stagusrf = su.data(); o.stagthck = sh.data();
  o.beta_internal = beta.data(); o.flwafact = fl.data(); o.active_cell = ac.data();
  o.active_vertex = av.data(); o.loadu = lu.data(); o.loadv = lv.data();
  o.umask_dirichlet = um.data(); o.vmask_dirichlet = vm.data();
  if (m->sliding) {
    o.f_ground = fg.data();
    o.flwa_basal_stag = fbs.data();
  }
  if (m->approx_2d == 3) {
    o.dusrf_dx = gx.data();
    o.dusrf_dy = gy.data();
  }
  if (m->approx_2d == 4) o.ice_plus_land_mask = iplm.data();
  bp_inputs in;
  const int rc = bp_setup(m, &o, uvel, vvel, &in);
  if (rc != BP_OK) return rc;
  return bp_solve(ctx, &in, uvel, vvel, efvs, stats);
}
