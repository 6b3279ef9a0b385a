/*
 * bp_oracle.c -- CPU restatement of CISM's Blatter-Pattyn velocity solve.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the B200 solver, never part of
 * the product path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load this library.
 *
 * Each function cites the reference routine it restates (paths relative to
 * the CISM source tree).  Loop order, constants, units (m, m/a, Pa a) and
 * the vol0 = 1e9 matrix scaling follow the Fortran, so results agree with
 * the reference to floating-point roundoff.  Arrays use the reference's
 * column-major layout with a 2-cell halo; indices below are 1-based.
 *
 * Parity pinning: the reference ships no golden vectors and its Fortran
 * cannot be compiled here (no Fortran compiler).  The oracle is pinned by
 * the reference's own invariants, the analytic first-order slab solution of
 * tests/slab/plotSlab.py:143-157 and standard-vs-Chronopoulos-Gear
 * agreement (tests/test_oracle.py).
 */
#include "bp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IC(i, j) (((size_t)(j) - 1) * (size_t)nx + ((size_t)(i) - 1))
#define IV(i, j) (((size_t)(j) - 1) * (size_t)(nx - 1) + ((size_t)(i) - 1))
#define IX(k, i, j) (IV(i, j) * (size_t)nz + ((size_t)(k) - 1))
#define IFL(k, i, j) (IC(i, j) * (size_t)(nz - 1) + ((size_t)(k) - 1))
#define IA(m, k, i, j) (IX(k, i, j) * 27 + ((size_t)(m) - 1))

/* indxA_3d(iA,jA,kA): iA fastest, diagonal = 14
 * (glissade_velo_higher.F90:599-619). */
static int indxA(int iA, int jA, int kA) {
  return 1 + (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1);
}

/* ---------------------------------------------------------------------
 * Finite-element tables, glissade_velo_higher_init
 * (glissade_velo_higher.F90:270-650).
 * ------------------------------------------------------------------- */
static double xqp[8], yqp[8], zqp[8], wqp[8];
static double phi3[8][8], dxr3[8][8], dyr3[8][8], dzr3[8][8]; /* [n][p] */
static double xqp2[4], yqp2[4], wqp2[4];
static double phi2[4][4], dxr2[4][4], dyr2[4][4];
static int ishift[8][8], jshift[8][8], kshift[8][8];
static int tables_ready = 0;

static void init_tables(void) {
  if (tables_ready) return;
  const double r = 1.0 / sqrt(3.0);
  const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  const double sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  const double sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int p = 0; p < 8; ++p) {
    xqp[p] = sx[p] * r; yqp[p] = sy[p] * r; zqp[p] = sz[p] * r; wqp[p] = 1.0;
  }
  for (int p = 0; p < 8; ++p) {
    double x = xqp[p], y = yqp[p], z = zqp[p];
    for (int n = 0; n < 8; ++n) {
      double ax = sx[n], ay = sy[n], az = sz[n];
      phi3[n][p] = (1.0 + ax * x) * (1.0 + ay * y) * (1.0 + az * z) / 8.0;
      dxr3[n][p] = ax * (1.0 + ay * y) * (1.0 + az * z) / 8.0;
      dyr3[n][p] = ay * (1.0 + ax * x) * (1.0 + az * z) / 8.0;
      dzr3[n][p] = az * (1.0 + ax * x) * (1.0 + ay * y) / 8.0;
    }
  }
  const double s2x[4] = {-1, 1, 1, -1}, s2y[4] = {-1, -1, 1, 1};
  for (int p = 0; p < 4; ++p) {
    xqp2[p] = s2x[p] * r; yqp2[p] = s2y[p] * r; wqp2[p] = 1.0;
  }
  for (int p = 0; p < 4; ++p)
    for (int n = 0; n < 4; ++n) {
      phi2[n][p] = (1.0 + s2x[n] * xqp2[p]) * (1.0 + s2y[n] * yqp2[p]) / 4.0;
      dxr2[n][p] = s2x[n] * (1.0 + s2y[n] * yqp2[p]) / 4.0;
      dyr2[n][p] = s2y[n] * (1.0 + s2x[n] * xqp2[p]) / 4.0;
    }
  /* ishift/jshift/kshift, glissade_velo_higher.F90:453-486 */
  const int i1[8] = {0, 1, 1, 0, 0, 1, 1, 0};
  const int i2[8] = {-1, 0, 0, -1, -1, 0, 0, -1};
  const int j1[8] = {0, 0, 1, 1, 0, 0, 1, 1};
  const int j3[8] = {-1, -1, 0, 0, -1, -1, 0, 0};
  const int k1[8] = {0, 0, 0, 0, -1, -1, -1, -1};
  const int k5[8] = {1, 1, 1, 1, 0, 0, 0, 0};
  const int irow[8] = {0, 1, 1, 0, 0, 1, 1, 0}; /* 0 -> i1, 1 -> i2 */
  const int jrow[8] = {0, 0, 1, 1, 0, 0, 1, 1}; /* 0 -> j1, 1 -> j3 */
  const int krow[8] = {0, 0, 0, 0, 1, 1, 1, 1}; /* 0 -> k1, 1 -> k5 */
  for (int n = 0; n < 8; ++n)
    for (int c = 0; c < 8; ++c) {
      ishift[n][c] = irow[n] ? i2[c] : i1[c];
      jshift[n][c] = jrow[n] ? j3[c] : j1[c];
      kshift[n][c] = krow[n] ? k5[c] : k1[c];
    }
  tables_ready = 1;
}

/* Glide sigma, glide_setup.F90:281-290 and 375-382 (which_sigma = 0). */
void orc_sigma_glide(int nz, double *sigma, double *stagwbndsigma) {
  for (int up = 1; up <= nz; ++up) {
    double level = (double)(up - 1) / (double)(nz - 1);
    sigma[up - 1] = (1.0 - pow(level + 1.0, -2.0)) / (1.0 - pow(2.0, -2.0));
  }
  if (stagwbndsigma) {
    stagwbndsigma[0] = 0.0;
    for (int k = 1; k <= nz - 1; ++k)
      stagwbndsigma[k] = (sigma[k - 1] + sigma[k]) / 2.0;
    stagwbndsigma[nz] = 1.0;
  }
}

/* ---------------------------------------------------------------------
 * Halo updates: parallel_slap.F90 parallel_halo_real8_2d (:1790-1860) and
 * staggered_parallel_halo_real8_3d/_4d (:2807-2925).  lhalo = uhalo = 2
 * for cells; staggered_lhalo = 2, staggered_uhalo = 1.
 * ------------------------------------------------------------------- */
void orc_halo_cell_real(int nx, int ny, int periodic, double *a,
                        double offset_ew, double offset_ns) {
  if (!periodic) {
    for (int j = 3; j <= ny - 2; ++j) {
      a[IC(1, j)] = a[IC(2, j)] = 0.0;
      a[IC(nx - 1, j)] = a[IC(nx, j)] = 0.0;
    }
    for (int i = 1; i <= nx; ++i) {
      a[IC(i, 1)] = a[IC(i, 2)] = 0.0;
      a[IC(i, ny - 1)] = a[IC(i, ny)] = 0.0;
    }
    return;
  }
  for (int j = 3; j <= ny - 2; ++j) {
    double e1 = a[IC(nx - 3, j)], e2 = a[IC(nx - 2, j)];
    double w1 = a[IC(3, j)], w2 = a[IC(4, j)];
    a[IC(1, j)] = e1 + offset_ew; a[IC(2, j)] = e2 + offset_ew;
    a[IC(nx - 1, j)] = w1 - offset_ew; a[IC(nx, j)] = w2 - offset_ew;
  }
  for (int i = 1; i <= nx; ++i) {
    double n1 = a[IC(i, ny - 3)], n2 = a[IC(i, ny - 2)];
    double s1 = a[IC(i, 3)], s2 = a[IC(i, 4)];
    a[IC(i, 1)] = n1 + offset_ns; a[IC(i, 2)] = n2 + offset_ns;
    a[IC(i, ny - 1)] = s1 - offset_ns; a[IC(i, ny)] = s2 - offset_ns;
  }
}

static void halo_cell_int(int nx, int ny, int periodic, int *a) {
  if (!periodic) {
    for (int j = 3; j <= ny - 2; ++j) {
      a[IC(1, j)] = a[IC(2, j)] = 0;
      a[IC(nx - 1, j)] = a[IC(nx, j)] = 0;
    }
    for (int i = 1; i <= nx; ++i) {
      a[IC(i, 1)] = a[IC(i, 2)] = 0;
      a[IC(i, ny - 1)] = a[IC(i, ny)] = 0;
    }
    return;
  }
  for (int j = 3; j <= ny - 2; ++j) {
    int e1 = a[IC(nx - 3, j)], e2 = a[IC(nx - 2, j)];
    int w1 = a[IC(3, j)], w2 = a[IC(4, j)];
    a[IC(1, j)] = e1; a[IC(2, j)] = e2;
    a[IC(nx - 1, j)] = w1; a[IC(nx, j)] = w2;
  }
  for (int i = 1; i <= nx; ++i) {
    int n1 = a[IC(i, ny - 3)], n2 = a[IC(i, ny - 2)];
    int s1 = a[IC(i, 3)], s2 = a[IC(i, 4)];
    a[IC(i, 1)] = n1; a[IC(i, 2)] = n2;
    a[IC(i, ny - 1)] = s1; a[IC(i, ny)] = s2;
  }
}

/* a has leading dimension nlead and trailing (nx-1, ny-1). */
void orc_halo_stag(int nx, int ny, int nlead, int periodic, double *a) {
  const int V = nx - 1, W = ny - 1;
#define AS(l, i, j) a[(((size_t)(j) - 1) * (size_t)V + ((size_t)(i) - 1)) * (size_t)nlead + (size_t)(l)]
  if (!periodic) {
    for (int j = 1; j <= W; ++j)
      for (int l = 0; l < nlead; ++l) { AS(l, 1, j) = 0.0; AS(l, V, j) = 0.0; }
    for (int i = 1; i <= V; ++i)
      for (int l = 0; l < nlead; ++l) { AS(l, i, 1) = 0.0; AS(l, i, W) = 0.0; }
    return;
  }
  for (int j = 3; j <= W - 1; ++j)
    for (int l = 0; l < nlead; ++l) {
      double wcp = AS(l, 3, j);
      double e1 = AS(l, V - 2, j), e2 = AS(l, V - 1, j);
      AS(l, V, j) = wcp;
      AS(l, 1, j) = e1;
      AS(l, 2, j) = e2;
    }
  for (int i = 1; i <= V; ++i)
    for (int l = 0; l < nlead; ++l) {
      double scp = AS(l, i, 3);
      double n1 = AS(l, i, W - 2), n2 = AS(l, i, W - 1);
      AS(l, i, W) = scp;
      AS(l, i, 1) = n1;
      AS(l, i, 2) = n2;
    }
#undef AS
}

/* Locally owned vertex range, parallel_slap.F90:655-673. */
static void owned_range(int nx, int ny, int periodic, int *ilo, int *ihi,
                        int *jlo, int *jhi) {
  *ilo = periodic ? 3 : 2;
  *jlo = periodic ? 3 : 2;
  *ihi = nx - 2;
  *jhi = ny - 2;
}

/* ---------------------------------------------------------------------
 * glissade_get_masks (glissade_masks.F90:55-457) with the default
 * which_ho_calving_front = NO_SUBGRID, so active_ice_mask = ice_mask and
 * calving_front_mask = 0.
 * ------------------------------------------------------------------- */
void orc_get_masks(int nx, int ny, int periodic, const double *thck,
                   const double *topg, double eus, double thklim,
                   double rhoi, double rhoo, int *ice_mask,
                   int *floating_mask, int *ocean_mask, int *land_mask,
                   int *active_ice_mask) {
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      size_t c = IC(i, j);
      ice_mask[c] = thck[c] > thklim ? 1 : 0;
      ocean_mask[c] = (topg[c] < eus && ice_mask[c] == 0) ? 1 : 0;
      floating_mask[c] =
          (topg[c] - eus < (-rhoi / rhoo) * thck[c] && ice_mask[c] == 1) ? 1 : 0;
      land_mask[c] = topg[c] >= eus ? 1 : 0;
      active_ice_mask[c] = ice_mask[c];
    }
  halo_cell_int(nx, ny, periodic, ice_mask);
  halo_cell_int(nx, ny, periodic, floating_mask);
  halo_cell_int(nx, ny, periodic, active_ice_mask);
}

/* glissade_stagger (glissade_grid_operators.F90:60-148). */
void orc_stagger(int nx, int ny, const double *var, double *stagvar,
                 const int *mask, int stagger_margin) {
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      size_t v = IV(i, j);
      stagvar[v] = 0.0;
      if (stagger_margin == 0) {
        stagvar[v] = (var[IC(i, j + 1)] + var[IC(i + 1, j + 1)] +
                      var[IC(i, j)] + var[IC(i + 1, j)]) / 4.0;
      } else {
        double sumvar = mask[IC(i, j + 1)] * var[IC(i, j + 1)] +
                        mask[IC(i + 1, j + 1)] * var[IC(i + 1, j + 1)] +
                        mask[IC(i, j)] * var[IC(i, j)] +
                        mask[IC(i + 1, j)] * var[IC(i + 1, j)];
        double summask = (double)(mask[IC(i, j + 1)] + mask[IC(i + 1, j + 1)] +
                                  mask[IC(i, j)] + mask[IC(i + 1, j)]);
        if (summask > 0.0) stagvar[v] = sumvar / summask;
      }
    }
}

/* Fortran MIN/MAX on a NaN operand: the finite operand is returned (IEEE
 * minNum/maxNum), which fmin/fmax implement. */
static double edge_ramp(double thck_upper, double thklim, double ramp) {
  double f = fmin(1.0, (thck_upper - thklim) / ramp);
  return fmax(f, 0.0);
}

/* glissade_surface_elevation_gradient (glissade_grid_operators.F90:734-1168),
 * centered gradient (which_ho_gradient = 0). */
void orc_surface_gradient(int nx, int ny, int periodic, double dx, double dy,
                          const int *active_ice_mask, const int *land_mask,
                          const double *usrf, const double *thck,
                          double thklim, double thck_gradient_ramp,
                          int ho_gradient, int ho_gradient_margin,
                          double max_slope, double *ds_dx, double *ds_dy) {
  double *ex = calloc((size_t)nx * ny, sizeof(double));
  double *ey = calloc((size_t)nx * ny, sizeof(double));
  if (ho_gradient_margin == ORC_GRADIENT_MARGIN_LAND) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        ex[IC(i, j)] = (usrf[IC(i + 1, j)] - usrf[IC(i, j)]) / dx;
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx; ++i)
        ey[IC(i, j)] = (usrf[IC(i, j + 1)] - usrf[IC(i, j)]) / dy;
  } else if (ho_gradient_margin == ORC_GRADIENT_MARGIN_MARINE) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        if (active_ice_mask[IC(i, j)] == 1 && active_ice_mask[IC(i + 1, j)] == 1)
          ex[IC(i, j)] = (usrf[IC(i + 1, j)] - usrf[IC(i, j)]) / dx;
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx; ++i)
        if (active_ice_mask[IC(i, j)] == 1 && active_ice_mask[IC(i, j + 1)] == 1)
          ey[IC(i, j)] = (usrf[IC(i, j + 1)] - usrf[IC(i, j)]) / dy;
  } else { /* HYBRID */
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        int iu, il; double sgn;
        if (usrf[IC(i, j)] > usrf[IC(i + 1, j)]) { iu = i; il = i + 1; sgn = -1.0; }
        else { iu = i + 1; il = i; sgn = 1.0; }
        double ef = 1.0;
        if (land_mask[IC(iu, j)] == 1)
          ef = edge_ramp(thck[IC(iu, j)], thklim, thck_gradient_ramp);
        if (active_ice_mask[IC(iu, j)] == 1 && active_ice_mask[IC(il, j)] == 1)
          ex[IC(i, j)] = ef * sgn * (usrf[IC(iu, j)] - usrf[IC(il, j)]) / dx;
        else if (active_ice_mask[IC(iu, j)] == 1 && land_mask[IC(il, j)] == 1)
          ex[IC(i, j)] = ef * sgn * (usrf[IC(iu, j)] - usrf[IC(il, j)]) / dx;
      }
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx; ++i) {
        int ju, jl; double sgn;
        if (usrf[IC(i, j)] > usrf[IC(i, j + 1)]) { ju = j; jl = j + 1; sgn = -1.0; }
        else { ju = j + 1; jl = j; sgn = 1.0; }
        double ef = 1.0;
        if (land_mask[IC(i, ju)] == 1)
          ef = edge_ramp(thck[IC(i, ju)], thklim, thck_gradient_ramp);
        if (active_ice_mask[IC(i, ju)] == 1 && active_ice_mask[IC(i, jl)] == 1)
          ey[IC(i, j)] = ef * sgn * (usrf[IC(i, ju)] - usrf[IC(i, jl)]) / dy;
        else if (active_ice_mask[IC(i, ju)] == 1 && land_mask[IC(i, jl)] == 1)
          ey[IC(i, j)] = ef * sgn * (usrf[IC(i, ju)] - usrf[IC(i, jl)]) / dy;
      }
  }
  memset(ds_dx, 0, (size_t)(nx - 1) * (ny - 1) * sizeof(double));
  memset(ds_dy, 0, (size_t)(nx - 1) * (ny - 1) * sizeof(double));
  if (ho_gradient == ORC_GRADIENT_CENTERED) {
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        ds_dx[IV(i, j)] = 0.5 * (ex[IC(i, j)] + ex[IC(i, j + 1)]);
        ds_dy[IV(i, j)] = 0.5 * (ey[IC(i, j)] + ey[IC(i + 1, j)]);
      }
  } else if (ho_gradient == ORC_GRADIENT_UPSTREAM1) {
    /* the edge on the higher side of the vertex (glissade_grid_operators.F90:1028-1058) */
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        double sum1 = usrf[IC(i, j + 1)] + usrf[IC(i + 1, j + 1)];
        double sum2 = usrf[IC(i, j)] + usrf[IC(i + 1, j)];
        ds_dx[IV(i, j)] = sum1 > sum2 ? ex[IC(i, j + 1)] : ex[IC(i, j)];
        sum1 = usrf[IC(i + 1, j)] + usrf[IC(i + 1, j + 1)];
        sum2 = usrf[IC(i, j)] + usrf[IC(i, j + 1)];
        ds_dy[IV(i, j)] = sum1 > sum2 ? ey[IC(i + 1, j)] : ey[IC(i, j)];
      }
  } else if (ho_gradient == ORC_GRADIENT_UPSTREAM2) {
    /* second order: two edges on the higher side (:1060-1093) */
    for (int j = 2; j <= ny - 2; ++j)
      for (int i = 2; i <= nx - 2; ++i) {
        double sum1 = usrf[IC(i, j + 1)] + usrf[IC(i + 1, j + 1)] + usrf[IC(i, j + 2)] + usrf[IC(i + 1, j + 2)];
        double sum2 = usrf[IC(i, j)] + usrf[IC(i + 1, j)] + usrf[IC(i, j - 1)] + usrf[IC(i + 1, j - 1)];
        ds_dx[IV(i, j)] = sum1 > sum2 ? 1.5 * ex[IC(i, j + 1)] - 0.5 * ex[IC(i, j + 2)]
                                      : 1.5 * ex[IC(i, j)] - 0.5 * ex[IC(i, j - 1)];
        sum1 = usrf[IC(i + 1, j)] + usrf[IC(i + 1, j + 1)] + usrf[IC(i + 2, j)] + usrf[IC(i + 2, j + 1)];
        sum2 = usrf[IC(i, j)] + usrf[IC(i, j + 1)] + usrf[IC(i - 1, j)] + usrf[IC(i - 1, j + 1)];
        ds_dy[IV(i, j)] = sum1 > sum2 ? 1.5 * ey[IC(i + 1, j)] - 0.5 * ey[IC(i + 2, j)]
                                      : 1.5 * ey[IC(i, j)] - 0.5 * ey[IC(i - 1, j)];
      }
  }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      size_t v = IV(i, j);
      ds_dx[v] = ds_dx[v] > 0.0 ? fmin(ds_dx[v], max_slope) : fmax(ds_dx[v], -max_slope);
      ds_dy[v] = ds_dy[v] > 0.0 ? fmin(ds_dy[v], max_slope) : fmax(ds_dy[v], -max_slope);
    }
  orc_halo_stag(nx, ny, 1, periodic, ds_dx);
  orc_halo_stag(nx, ny, 1, periodic, ds_dy);
  free(ex);
  free(ey);
}

/* glissade_grounded_fraction (glissade_grounding_line.F90:55-178).  The
 * vmask test reads land_mask(i+1,j+1) twice and never land_mask(i+1,j)
 * (:117); restated verbatim. */
void orc_grounded_fraction(int nx, int ny, const int *ice_mask,
                           const int *floating_mask, const int *land_mask,
                           int whichground, double *f_ground) {
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      int vm = ice_mask[IC(i, j + 1)] == 1 || ice_mask[IC(i + 1, j + 1)] == 1 ||
               ice_mask[IC(i, j)] == 1 || ice_mask[IC(i + 1, j)] == 1 ||
               land_mask[IC(i, j + 1)] == 1 || land_mask[IC(i + 1, j + 1)] == 1 ||
               land_mask[IC(i, j)] == 1 || land_mask[IC(i + 1, j + 1)] == 1;
      size_t v = IV(i, j);
      f_ground[v] = 0.0;
      if (!vm) continue;
      if (whichground == ORC_GROUND_ALL) { f_ground[v] = 1.0; continue; }
#define CG(a, b) ((ice_mask[IC(a, b)] == 1 && floating_mask[IC(a, b)] == 0) || land_mask[IC(a, b)] == 1)
      if (CG(i, j + 1) || CG(i + 1, j + 1) || CG(i, j) || CG(i + 1, j))
        f_ground[v] = 1.0;
#undef CG
    }
}

/* ---------------------------------------------------------------------
 * get_basis_function_derivatives_3d (glissade_velo_higher.F90:6360-6579)
 * ------------------------------------------------------------------- */
static int basis_derivs_3d(const double *x, const double *y, const double *z,
                           int p, double *dx, double *dy, double *dz,
                           double *detJ) {
  double J[3][3] = {{0}};
  for (int n = 0; n < 8; ++n) {
    J[0][0] = J[0][0] + dxr3[n][p] * x[n];
    J[0][1] = J[0][1] + dxr3[n][p] * y[n];
    J[0][2] = J[0][2] + dxr3[n][p] * z[n];
    J[1][0] = J[1][0] + dyr3[n][p] * x[n];
    J[1][1] = J[1][1] + dyr3[n][p] * y[n];
    J[1][2] = J[1][2] + dyr3[n][p] * z[n];
    J[2][0] = J[2][0] + dzr3[n][p] * x[n];
    J[2][1] = J[2][1] + dzr3[n][p] * y[n];
    J[2][2] = J[2][2] + dzr3[n][p] * z[n];
  }
  double cf[3][3];
  cf[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  cf[0][1] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]);
  cf[0][2] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  cf[1][0] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]);
  cf[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  cf[1][2] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]);
  cf[2][0] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  cf[2][1] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]);
  cf[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  double d = J[0][0] * cf[0][0] + J[0][1] * cf[0][1] + J[0][2] * cf[0][2];
  *detJ = d;
  if (!(fabs(d) > 0.0)) return ORC_ERR_SINGULAR_JAC;
  double Ji[3][3];
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) Ji[row][col] = cf[col][row] / d;
  for (int n = 0; n < 8; ++n) {
    dx[n] = Ji[0][0] * dxr3[n][p] + Ji[0][1] * dyr3[n][p] + Ji[0][2] * dzr3[n][p];
    dy[n] = Ji[1][0] * dxr3[n][p] + Ji[1][1] * dyr3[n][p] + Ji[1][2] * dzr3[n][p];
    dz[n] = Ji[2][0] * dxr3[n][p] + Ji[2][1] * dyr3[n][p] + Ji[2][2] * dzr3[n][p];
  }
  return ORC_OK;
}

/* get_basis_function_derivatives_2d (:6583-6751), detJ only is used. */
static int basis_detJ_2d(const double *x, const double *y, int p,
                         double *detJ) {
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
  for (int n = 0; n < 4; ++n) {
    J11 = J11 + dxr2[n][p] * x[n];
    J12 = J12 + dxr2[n][p] * y[n];
    J21 = J21 + dyr2[n][p] * x[n];
    J22 = J22 + dyr2[n][p] * y[n];
  }
  *detJ = J11 * J22 - J12 * J21;
  return fabs(*detJ) > 0.0 ? ORC_OK : ORC_ERR_SINGULAR_JAC;
}

/* compute_effective_viscosity, BP branch (:7199-7378). */
static double effective_viscosity(int whichefvs, double efvs_constant,
                                  const double *dx, const double *dy,
                                  const double *dz, const double *u,
                                  const double *v, double flwafact) {
  const double effstrain_min = 1.0e-8;
  const double p_effstr = (1.0 - 3.0) / 3.0;
  const double p2_effstr = p_effstr / 2.0;
  if (whichefvs == ORC_EFVS_CONSTANT) return efvs_constant;
  if (whichefvs == ORC_EFVS_FLOWFACT) {
    const double scyr = 31536000.0;
    double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    return flwafact * pow(effstrain, p_effstr);
  }
  double ux = 0, uy = 0, uz = 0, vx = 0, vy = 0, vz = 0;
  for (int n = 0; n < 8; ++n) {
    ux = ux + dx[n] * u[n];
    uy = uy + dy[n] * u[n];
    uz = uz + dz[n] * u[n];
    vx = vx + dx[n] * v[n];
    vy = vy + dy[n] * v[n];
    vz = vz + dz[n] * v[n];
  }
  double sq = effstrain_min * effstrain_min +
              (ux * ux + vy * vy + ux * vy + 0.25 * ((vx + uy) * (vx + uy))) +
              0.25 * (uz * uz + vz * vz);
  return flwafact * pow(sq, p2_effstr);
}

/* assemble_stiffness_matrix_3d (:4954-5204) with compute_element_matrix
 * (:7868-7986), check_symmetry_element_matrix (:9468-9529) and
 * element_to_global_matrix_3d (:7990-8054). */
int orc_assemble_3d(int nx, int ny, int nz, int nhalo, const double *sigma,
                    const int *active_cell, const double *xVertex,
                    const double *yVertex, const double *uvel,
                    const double *vvel, const double *stagusrf,
                    const double *stagthck, const double *flwafact,
                    int whichefvs, double efvs_constant, double *efvs,
                    double *Auu, double *Auv, double *Avu, double *Avv) {
  init_tables();
  const double vol0 = 1.0e9;
  size_t nA = (size_t)27 * nz * (nx - 1) * (ny - 1);
  memset(Auu, 0, nA * sizeof(double));
  memset(Auv, 0, nA * sizeof(double));
  memset(Avu, 0, nA * sizeof(double));
  memset(Avv, 0, nA * sizeof(double));
  memset(efvs, 0, (size_t)(nz - 1) * nx * ny * sizeof(double));
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!active_cell[IC(i, j)]) continue;
      for (int k = 1; k <= nz - 1; ++k) {
        double Kuu[8][8] = {{0}}, Kuv[8][8] = {{0}}, Kvu[8][8] = {{0}},
               Kvv[8][8] = {{0}};
        double x[8], y[8], z[8], u[8], v[8];
        for (int n = 0; n < 8; ++n) {
          int in = i + ishift[6][n], jn = j + jshift[6][n], kn = k + kshift[6][n];
          x[n] = xVertex[IV(in, jn)];
          y[n] = yVertex[IV(in, jn)];
          z[n] = stagusrf[IV(in, jn)] - sigma[kn - 1] * stagthck[IV(in, jn)];
          u[n] = uvel[IX(kn, in, jn)];
          v[n] = vvel[IX(kn, in, jn)];
        }
        double efvs_qp[8];
        for (int p = 0; p < 8; ++p) {
          double ddx[8], ddy[8], ddz[8], detJ;
          if (basis_derivs_3d(x, y, z, p, ddx, ddy, ddz, &detJ) != ORC_OK)
            return ORC_ERR_SINGULAR_JAC;
          efvs_qp[p] = effective_viscosity(whichefvs, efvs_constant, ddx, ddy,
                                           ddz, u, v, flwafact[IFL(k, i, j)]);
          double f = efvs_qp[p] * wqp[p] * detJ / vol0;
          for (int nc = 0; nc < 8; ++nc)
            for (int nr = 0; nr < 8; ++nr) {
              Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * ddx[nr] * ddx[nc] +
                                               ddy[nr] * ddy[nc] + ddz[nr] * ddz[nc]);
              Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * ddx[nr] * ddy[nc] + ddy[nr] * ddx[nc]);
              Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * ddy[nr] * ddx[nc] + ddx[nr] * ddy[nc]);
              Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * ddy[nr] * ddy[nc] +
                                               ddx[nr] * ddx[nc] + ddz[nr] * ddz[nc]);
            }
        }
        double e = 0.0;
        for (int p = 0; p < 8; ++p) e = e + efvs_qp[p];
        efvs[IFL(k, i, j)] = e / 8.0;
        /* check_symmetry_element_matrix: eps10 absolute */
        for (int a = 0; a < 8; ++a)
          for (int b = 0; b < 8; ++b) {
            if (fabs(Kuu[a][b] - Kuu[b][a]) > 1.0e-10) return ORC_ERR_ASYMMETRIC_ELEMENT;
            if (fabs(Kvv[a][b] - Kvv[b][a]) > 1.0e-10) return ORC_ERR_ASYMMETRIC_ELEMENT;
            if (fabs(Kuv[a][b] - Kvu[b][a]) > 1.0e-10) return ORC_ERR_ASYMMETRIC_ELEMENT;
          }
        for (int nr = 0; nr < 8; ++nr) {
          int ii = i + ishift[6][nr], jj = j + jshift[6][nr], kk = k + kshift[6][nr];
          for (int nc = 0; nc < 8; ++nc) {
            int m = indxA(ishift[nr][nc], jshift[nr][nc], kshift[nr][nc]);
            size_t a = IA(m, kk, ii, jj);
            Auu[a] = Auu[a] + Kuu[nr][nc];
            Auv[a] = Auv[a] + Kuv[nr][nc];
            Avu[a] = Avu[a] + Kvu[nr][nc];
            Avv[a] = Avv[a] + Kvv[nr][nc];
          }
        }
      }
    }
  return ORC_OK;
}

/* compute_internal_stress (glissade_velo_higher.F90:6968-7195), 3-D
 * higher-order branch: at every element of an active cell, the strain
 * rates and the effective viscosity at the 8 quadrature points of the given
 * velocity, averaged; tau_eff from the averaged components. */
int orc_internal_stress(int nx, int ny, int nz, int nhalo, const double *sigma,
                        const int *active_cell, const double *xVertex,
                        const double *yVertex, const double *stagusrf,
                        const double *stagthck, const double *flwafact,
                        int whichefvs, double efvs_constant, const double *uvel,
                        const double *vvel, double *tau_xz, double *tau_yz,
                        double *tau_xx, double *tau_yy, double *tau_xy,
                        double *tau_eff) {
  return orc_internal_stress_approx(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex,
                                    stagusrf, stagthck, flwafact, NULL, whichefvs, efvs_constant,
                                    ORC_APPROX_BP, uvel, vvel, tau_xz, tau_yz, tau_xx, tau_yy,
                                    tau_xy, tau_eff);
}

/* compute_internal_stress for approximation approx (:7100-7147): the SSA
 * takes the horizontal gradients only and its viscosity branch
 * (:7325-7338); L1L2 takes the element's layer viscosity efvs(k,i,j) at
 * every point; Blatter-Pattyn and DIVA the 3-D gradients and viscosity. */
int orc_internal_stress_approx(int nx, int ny, int nz, int nhalo, const double *sigma,
                               const int *active_cell, const double *xVertex,
                               const double *yVertex, const double *stagusrf,
                               const double *stagthck, const double *flwafact,
                               const double *efvs, int whichefvs, double efvs_constant,
                               int approx, const double *uvel, const double *vvel,
                               double *tau_xz, double *tau_yz, double *tau_xx, double *tau_yy,
                               double *tau_xy, double *tau_eff) {
  init_tables();
  const size_t ne = (size_t)(nz - 1) * nx * ny;
  memset(tau_xz, 0, ne * sizeof(double));
  memset(tau_yz, 0, ne * sizeof(double));
  memset(tau_xx, 0, ne * sizeof(double));
  memset(tau_yy, 0, ne * sizeof(double));
  memset(tau_xy, 0, ne * sizeof(double));
  memset(tau_eff, 0, ne * sizeof(double));
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!active_cell[IC(i, j)]) continue;
      for (int k = 1; k <= nz - 1; ++k) {
        double x[8], y[8], z[8], u[8], v[8];
        for (int n = 0; n < 8; ++n) {
          int in = i + ishift[6][n], jn = j + jshift[6][n], kn = k + kshift[6][n];
          x[n] = xVertex[IV(in, jn)];
          y[n] = yVertex[IV(in, jn)];
          z[n] = stagusrf[IV(in, jn)] - sigma[kn - 1] * stagthck[IV(in, jn)];
          u[n] = uvel[IX(kn, in, jn)];
          v[n] = vvel[IX(kn, in, jn)];
        }
        const size_t e = IFL(k, i, j);
        for (int p = 0; p < 8; ++p) {
          double ddx[8], ddy[8], ddz[8], detJ;
          if (basis_derivs_3d(x, y, z, p, ddx, ddy, ddz, &detJ) != ORC_OK)
            return ORC_ERR_SINGULAR_JAC;
          double du_dx = 0.0, du_dy = 0.0, du_dz = 0.0, dv_dx = 0.0, dv_dy = 0.0, dv_dz = 0.0;
          for (int n = 0; n < 8; ++n) {
            du_dx = du_dx + ddx[n] * u[n];
            du_dy = du_dy + ddy[n] * u[n];
            du_dz = du_dz + ddz[n] * u[n];
            dv_dx = dv_dx + ddx[n] * v[n];
            dv_dy = dv_dy + ddy[n] * v[n];
            dv_dz = dv_dz + ddz[n] * v[n];
          }
          double efvs_qp;
          if (approx == ORC_APPROX_SSA) {
            du_dz = 0.0;
            dv_dz = 0.0;
            if (whichefvs == ORC_EFVS_NONLINEAR) {
              const double sq = 1.0e-8 * 1.0e-8 + (du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy +
                                                   0.25 * ((dv_dx + du_dy) * (dv_dx + du_dy)));
              efvs_qp = flwafact[e] * pow(sq, ((1.0 - 3.0) / 3.0) / 2.0);
            } else {
              efvs_qp = effective_viscosity(whichefvs, efvs_constant, ddx, ddy, ddz, u, v, flwafact[e]);
            }
          } else if (approx == ORC_APPROX_L1L2) {
            efvs_qp = efvs[e];
          } else {
            efvs_qp = effective_viscosity(whichefvs, efvs_constant, ddx, ddy, ddz, u, v, flwafact[e]);
          }
          tau_xz[e] = tau_xz[e] + efvs_qp * du_dz;
          tau_yz[e] = tau_yz[e] + efvs_qp * dv_dz;
          tau_xx[e] = tau_xx[e] + 2.0 * efvs_qp * du_dx;
          tau_yy[e] = tau_yy[e] + 2.0 * efvs_qp * dv_dy;
          tau_xy[e] = tau_xy[e] + efvs_qp * (dv_dx + du_dy);
        }
        tau_xz[e] = tau_xz[e] / 8;
        tau_yz[e] = tau_yz[e] / 8;
        tau_xx[e] = tau_xx[e] / 8;
        tau_yy[e] = tau_yy[e] / 8;
        tau_xy[e] = tau_xy[e] / 8;
        tau_eff[e] = sqrt(tau_xx[e] * tau_xx[e] + tau_yy[e] * tau_yy[e] + tau_xx[e] * tau_yy[e] +
                          tau_xy[e] * tau_xy[e] + tau_xz[e] * tau_xz[e] + tau_yz[e] * tau_yz[e]);
      }
    }
  return ORC_OK;
}

/* compute_basal_friction_heatflx (:6755-6964): the frictional heat flux
 * beta |u_b|^2 / scyr (W/m^2) at cell centres from the basal velocity
 * (uvel, vvel)(nz,:,:), by the 2x2 face quadrature over active cells
 * (which = 0) or at active vertices and unstaggered to cells with
 * glissade_unstagger margin 0 (which = 1, glissade_grid_operators.F90:
 * 152-231); then the cell halo update. */
void orc_basal_friction_heatflx(int nx, int ny, int nz, int nhalo, int periodic,
                                const int *active_cell, const int *active_vertex,
                                const double *uvel, const double *vvel,
                                const double *beta, int which, double *bfricflx) {
  init_tables();
  const double scyr = 31536000.0;
  memset(bfricflx, 0, (size_t)nx * ny * sizeof(double));
  if (which == 0) {
    for (int j = nhalo + 1; j <= ny - nhalo; ++j)
      for (int i = nhalo + 1; i <= nx - nhalo; ++i) {
        if (!active_cell[IC(i, j)]) continue;
        double u[4], v[4], b[4];
        for (int n = 0; n < 4; ++n) {
          const int iv = i + ishift[2][n], jv = j + jshift[2][n];
          u[n] = uvel[IX(nz, iv, jv)];
          v[n] = vvel[IX(nz, iv, jv)];
          b[n] = beta[IV(iv, jv)];
        }
        double sum_wqp = 0.0;
        for (int p = 0; p < 4; ++p) {
          double u_qp = 0.0, v_qp = 0.0, beta_qp = 0.0;
          for (int n = 0; n < 4; ++n) {
            u_qp = u_qp + phi2[n][p] * u[n];
            v_qp = v_qp + phi2[n][p] * v[n];
            beta_qp = beta_qp + phi2[n][p] * b[n];
          }
          bfricflx[IC(i, j)] = bfricflx[IC(i, j)] + wqp2[p] * beta_qp * (u_qp * u_qp + v_qp * v_qp);
          sum_wqp = sum_wqp + wqp2[p];
        }
        bfricflx[IC(i, j)] = bfricflx[IC(i, j)] / (sum_wqp * scyr);
      }
  } else {
    double *stag = calloc((size_t)(nx - 1) * (ny - 1), sizeof(double));
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        if (!active_vertex[IV(i, j)]) continue;
        const double ub = uvel[IX(nz, i, j)], vb = vvel[IX(nz, i, j)];
        stag[IV(i, j)] = beta[IV(i, j)] * (ub * ub + vb * vb);
        stag[IV(i, j)] = stag[IV(i, j)] / scyr;
      }
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        bfricflx[IC(i, j)] = (stag[IV(i, j)] + stag[IV(i - 1, j)] + stag[IV(i, j - 1)] +
                              stag[IV(i - 1, j - 1)]) / 4.0;
    free(stag);
  }
  orc_halo_cell_real(nx, ny, periodic, bfricflx, 0.0, 0.0);
}

/* basal_sliding_bc (:8125-8381) applied to the bed layer (k = nz). */
static void basal_sliding_bc(int nx, int ny, int nz, int nhalo, double dx,
                             double dy, const int *active_cell,
                             const int *active_vertex, const double *beta,
                             const double *xVertex, const double *yVertex,
                             int whichassemble_beta, double *Auu,
                             double *Avv) {
  const double vol0 = 1.0e9;
  if (whichassemble_beta == ORC_ASSEMBLE_LOCAL) {
    int m = indxA(0, 0, 0);
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        if (active_vertex[IV(i, j)]) {
          Auu[IA(m, nz, i, j)] = Auu[IA(m, nz, i, j)] + dx * dy / vol0 * beta[IV(i, j)];
          Avv[IA(m, nz, i, j)] = Avv[IA(m, nz, i, j)] + dx * dy / vol0 * beta[IV(i, j)];
        }
    return;
  }
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!active_cell[IC(i, j)]) continue;
      double x[4] = {xVertex[IV(i - 1, j - 1)], xVertex[IV(i, j - 1)],
                     xVertex[IV(i, j)], xVertex[IV(i - 1, j)]};
      double y[4] = {yVertex[IV(i - 1, j - 1)], yVertex[IV(i, j - 1)],
                     yVertex[IV(i, j)], yVertex[IV(i - 1, j)]};
      double b[4] = {beta[IV(i - 1, j - 1)], beta[IV(i, j - 1)],
                     beta[IV(i, j)], beta[IV(i - 1, j)]};
      for (int p = 0; p < 4; ++p) {
        double detJ;
        basis_detJ_2d(x, y, p, &detJ);
        double bq = 0.0;
        for (int n = 0; n < 4; ++n) bq = bq + phi2[n][p] * b[n];
        double K[4][4];
        for (int nc = 0; nc < 4; ++nc)
          for (int nr = 0; nr < 4; ++nr)
            K[nr][nc] = 0.0 + bq * wqp2[p] * detJ / vol0 * phi2[nr][p] * phi2[nc][p];
        for (int nr = 0; nr < 4; ++nr) {
          int ii = i + ishift[2][nr], jj = j + jshift[2][nr];
          for (int nc = 0; nc < 4; ++nc) {
            int m = indxA(ishift[nr][nc], jshift[nr][nc], 0);
            Auu[IA(m, nz, ii, jj)] = Auu[IA(m, nz, ii, jj)] + K[nr][nc];
            Avv[IA(m, nz, ii, jj)] = Avv[IA(m, nz, ii, jj)] + K[nr][nc];
          }
        }
      }
    }
}

/* dirichlet_boundary_conditions_3d (:8385-8578). */
static void dirichlet_bc_3d(int nx, int ny, int nz, int nhalo,
                            const int *active_vertex, const int *umask,
                            const int *vmask, const double *uvel,
                            const double *vvel, double *Auu, double *Auv,
                            double *Avu, double *Avv, double *bu,
                            double *bv) {
  for (int j = nhalo; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo; i <= nx - nhalo + 1; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      for (int k = 1; k <= nz; ++k) {
        if (umask[IX(k, i, j)] == 1) {
          bu[IX(k, i, j)] = uvel[IX(k, i, j)];
          for (int kA = -1; kA <= 1; ++kA)
            for (int jA = -1; jA <= 1; ++jA)
              for (int iA = -1; iA <= 1; ++iA) {
                if (!(k + kA >= 1 && k + kA <= nz && i + iA >= 1 && i + iA <= nx - 1 &&
                      j + jA >= 1 && j + jA <= ny - 1)) continue;
                if (iA == 0 && jA == 0 && kA == 0) {
                  int m = indxA(0, 0, 0);
                  Auu[IA(m, k, i, j)] = 1.0;
                  Auv[IA(m, k, i, j)] = 0.0;
                  Avu[IA(m, k, i, j)] = 0.0;
                } else {
                  int m = indxA(iA, jA, kA);
                  Auu[IA(m, k, i, j)] = 0.0;
                  Auv[IA(m, k, i, j)] = 0.0;
                  int mm = indxA(-iA, -jA, -kA);
                  size_t nb = IX(k + kA, i + iA, j + jA);
                  size_t an = IA(mm, k + kA, i + iA, j + jA);
                  if (umask[nb] != 1) {
                    bu[nb] = bu[nb] - Auu[an] * uvel[IX(k, i, j)];
                    Auu[an] = 0.0;
                  }
                  if (vmask[nb] != 1) {
                    bv[nb] = bv[nb] - Avu[an] * uvel[IX(k, i, j)];
                    Avu[an] = 0.0;
                  }
                }
              }
        }
        if (vmask[IX(k, i, j)] == 1) {
          bv[IX(k, i, j)] = vvel[IX(k, i, j)];
          for (int kA = -1; kA <= 1; ++kA)
            for (int jA = -1; jA <= 1; ++jA)
              for (int iA = -1; iA <= 1; ++iA) {
                if (!(k + kA >= 1 && k + kA <= nz && i + iA >= 1 && i + iA <= nx - 1 &&
                      j + jA >= 1 && j + jA <= ny - 1)) continue;
                if (iA == 0 && jA == 0 && kA == 0) {
                  int m = indxA(0, 0, 0);
                  Auv[IA(m, k, i, j)] = 0.0;
                  Avu[IA(m, k, i, j)] = 0.0;
                  Avv[IA(m, k, i, j)] = 1.0;
                } else {
                  int m = indxA(iA, jA, kA);
                  Avu[IA(m, k, i, j)] = 0.0;
                  Avv[IA(m, k, i, j)] = 0.0;
                  int mm = indxA(-iA, -jA, -kA);
                  size_t nb = IX(k + kA, i + iA, j + jA);
                  size_t an = IA(mm, k + kA, i + iA, j + jA);
                  if (umask[nb] != 1) {
                    bu[nb] = bu[nb] - Auv[an] * vvel[IX(k, i, j)];
                    Auv[an] = 0.0;
                  }
                  if (vmask[nb] != 1) {
                    bv[nb] = bv[nb] - Avv[an] * vvel[IX(k, i, j)];
                    Avv[an] = 0.0;
                  }
                }
              }
        }
      }
    }
}

/* check_symmetry_assembled_matrix_3d (:9533-9741). */
static void check_symmetry_assembled_3d(int nx, int ny, int nz, int periodic,
                                        const int *active_vertex, double *Auu,
                                        double *Auv, double *Avu,
                                        double *Avv) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  const double eps08 = 1.0e-8;
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      for (int k = 1; k <= nz; ++k) {
        for (int pass = 0; pass < 2; ++pass) {
          double *D = pass == 0 ? Auu : Avv;   /* block that owns the diag */
          double *O1 = pass == 0 ? Auv : Avu;  /* off-diagonal block, row */
          double *O2 = pass == 0 ? Avu : Auv;  /* its transpose partner */
          double diag = D[IA(indxA(0, 0, 0), k, i, j)];
          for (int jA = -1; jA <= 1; ++jA)
            for (int iA = -1; iA <= 1; ++iA)
              for (int kA = -1; kA <= 1; ++kA) {
                if (!(k + kA >= 1 && k + kA <= nz)) continue;
                int m = indxA(iA, jA, kA), mm = indxA(-iA, -jA, -kA);
                size_t a1 = IA(m, k, i, j), a2 = IA(mm, k + kA, i + iA, j + jA);
                double v1 = D[a1], v2 = D[a2];
                if (v2 != v1 && fabs(v2 - v1) < eps08 * fabs(diag)) {
                  double avg = 0.5 * (v1 + v2);
                  D[a1] = avg;
                  D[a2] = avg;
                }
                v1 = O1[a1];
                v2 = O2[a2];
                if (v2 != v1 && fabs(v2 - v1) < eps08 * fabs(diag)) {
                  double avg = 0.5 * (v1 + v2);
                  O1[a1] = avg;
                  O2[a2] = avg;
                }
              }
        }
      }
    }
}

/* count_nonzeros_3d (:9355-9410). */
static long count_nonzeros_3d(int nx, int ny, int nz, int periodic,
                              const int *active_vertex, const double *Auu,
                              const double *Auv, const double *Avu,
                              const double *Avv) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  long nnz = 0;
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      for (int k = 1; k <= nz; ++k)
        for (int m = 1; m <= 27; ++m) {
          size_t a = IA(m, k, i, j);
          nnz += (Auu[a] != 0.0) + (Auv[a] != 0.0) + (Avu[a] != 0.0) + (Avv[a] != 0.0);
        }
    }
  return nnz;
}

/* matvec_multiply_structured_3d (glissade_velo_higher_pcg.F90:2533-2647). */
void orc_matvec_3d(int nx, int ny, int nz, int periodic,
                   const int *active_vertex, const double *Auu,
                   const double *Auv, const double *Avu, const double *Avv,
                   const double *xu, const double *xv, double *yu,
                   double *yv) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  size_t nv = (size_t)nz * (nx - 1) * (ny - 1);
  memset(yu, 0, nv * sizeof(double));
  memset(yv, 0, nv * sizeof(double));
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      for (int k = 1; k <= nz; ++k) {
        double su = 0.0, sv = 0.0;
        for (int kA = -1; kA <= 1; ++kA)
          for (int jA = -1; jA <= 1; ++jA)
            for (int iA = -1; iA <= 1; ++iA) {
              if (!(k + kA >= 1 && k + kA <= nz && i + iA >= 1 && i + iA <= nx - 1 &&
                    j + jA >= 1 && j + jA <= ny - 1)) continue;
              int m = indxA(iA, jA, kA);
              size_t a = IA(m, k, i, j), x = IX(k + kA, i + iA, j + jA);
              su = su + Auu[a] * xu[x] + Auv[a] * xv[x];
              sv = sv + Avu[a] * xu[x] + Avv[a] * xv[x];
            }
        yu[IX(k, i, j)] = su;
        yv[IX(k, i, j)] = sv;
      }
    }
}

/* global_sum_staggered_3d_real8 (:2333-2375): owned vertices only. */
static double gsum2(int nx, int ny, int nz, int periodic, const double *a1,
                    const double *b1, const double *a2, const double *b2) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  double s = 0.0;
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i)
      for (int k = 1; k <= nz; ++k) {
        size_t x = IX(k, i, j);
        double w1 = a1[x] * b1[x];
        double w2 = a2[x] * b2[x];
        s = s + w1 + w2;
      }
  return s;
}

/* setup_preconditioner_3d (:2150-2265) + diagonal / SIA application. */
typedef struct {
  int precond;
  double *Adiagu, *Adiagv; /* nz,nx-1,ny-1 */
  double *Muu, *Mvv;       /* (-1:1,nz,nx-1,ny-1) */
} precond_t;

static void setup_precond(int nx, int ny, int nz, int precond,
                          const double *Auu, const double *Avv,
                          precond_t *pc) {
  size_t nv = (size_t)nz * (nx - 1) * (ny - 1);
  pc->precond = precond;
  pc->Adiagu = calloc(nv, sizeof(double));
  pc->Adiagv = calloc(nv, sizeof(double));
  pc->Muu = calloc(3 * nv, sizeof(double));
  pc->Mvv = calloc(3 * nv, sizeof(double));
  for (size_t x = 0; x < nv; ++x) {
    if (precond == ORC_PRECOND_DIAG) {
      pc->Adiagu[x] = Auu[x * 27 + 13];
      pc->Adiagv[x] = Avv[x * 27 + 13];
    } else if (precond == ORC_PRECOND_SIA) {
      for (int d = 0; d < 3; ++d) {
        int m = indxA(0, 0, d - 1);
        pc->Muu[x * 3 + d] = Auu[x * 27 + (m - 1)];
        pc->Mvv[x * 3 + d] = Avv[x * 27 + (m - 1)];
      }
    }
  }
}

static void free_precond(precond_t *pc) {
  free(pc->Adiagu); free(pc->Adiagv); free(pc->Muu); free(pc->Mvv);
}

/* easy_sia_solver + tridiag_solver (:2759-2904). */
static void easy_sia_solver(int nx, int ny, int nz, const int *active_vertex,
                            const double *M, const double *b, double *x) {
  double *gamma = malloc((size_t)nz * sizeof(double));
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      const double *Mc = M + IX(1, i, j) * 3;
      const double *r = b + IX(1, i, j);
      double *s = x + IX(1, i, j);
      /* sbdiag(k) = M(-1,k), diag = M(0,k), spdiag = M(1,k); ends zeroed */
      double beta = Mc[1];
      s[0] = r[0] / beta;
      for (int k = 2; k <= nz; ++k) {
        double spd = (k - 1 == nz) ? 0.0 : Mc[(k - 2) * 3 + 2];
        double sbd = Mc[(k - 1) * 3 + 0];
        gamma[k - 1] = spd / beta;
        beta = Mc[(k - 1) * 3 + 1] - sbd * gamma[k - 1];
        s[k - 1] = (r[k - 1] - sbd * s[k - 2]) / beta;
      }
      for (int k = nz - 1; k >= 1; --k) s[k - 1] = s[k - 1] - gamma[k] * s[k];
    }
  free(gamma);
}

static void apply_precond(int nx, int ny, int nz, const precond_t *pc,
                          const int *active_vertex, const double *ru,
                          const double *rv, double *zu, double *zv) {
  size_t nv = (size_t)nz * (nx - 1) * (ny - 1);
  if (pc->precond == ORC_PRECOND_NONE) {
    memcpy(zu, ru, nv * sizeof(double));
    memcpy(zv, rv, nv * sizeof(double));
  } else if (pc->precond == ORC_PRECOND_DIAG) {
    for (size_t x = 0; x < nv; ++x) {
      zu[x] = pc->Adiagu[x] != 0.0 ? ru[x] / pc->Adiagu[x] : 0.0;
      zv[x] = pc->Adiagv[x] != 0.0 ? rv[x] / pc->Adiagv[x] : 0.0;
    }
  } else {
    easy_sia_solver(nx, ny, nz, active_vertex, pc->Muu, ru, zu);
    easy_sia_solver(nx, ny, nz, active_vertex, pc->Mvv, rv, zv);
  }
}

/* pcg_solver_standard_3d (glissade_velo_higher_pcg.F90:84-549); maxiters,
 * tolerance and solve_ncheck are parameters here (hard-coded 200, 1e-8, 5
 * in the reference, :67-77). */
int orc_pcg_standard_3d(int nx, int ny, int nz, int periodic,
                        const int *active_vertex, const double *Auu,
                        const double *Auv, const double *Avu,
                        const double *Avv, const double *bu, const double *bv,
                        double *xu, double *xv, int precond, int maxiters,
                        double tolerance, int ncheck, double *err,
                        int *niters) {
  size_t nv = (size_t)nz * (nx - 1) * (ny - 1);
  double *ru = calloc(nv, 8), *rv = calloc(nv, 8), *du = calloc(nv, 8),
         *dv = calloc(nv, 8), *qu = calloc(nv, 8), *qv = calloc(nv, 8),
         *zu = calloc(nv, 8), *zv = calloc(nv, 8);
  precond_t pc;
  setup_precond(nx, ny, nz, precond, Auu, Avv, &pc);
  orc_halo_stag(nx, ny, nz, periodic, xu);
  orc_halo_stag(nx, ny, nz, periodic, xv);
  orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, xu, xv, zu, zv);
  for (size_t x = 0; x < nv; ++x) { ru[x] = bu[x] - zu[x]; rv[x] = bv[x] - zv[x]; }
  *niters = maxiters;
  *err = -1.0;
  double eta0 = 1.0;
  memset(du, 0, nv * 8); memset(dv, 0, nv * 8);
  memset(zu, 0, nv * 8); memset(zv, 0, nv * 8);
  double L2_rhs = sqrt(gsum2(nx, ny, nz, periodic, bu, bu, bv, bv));
  int status = ORC_WARN_PCG_NOT_CONVERGED;
  for (int n = 1; n <= maxiters; ++n) {
    apply_precond(nx, ny, nz, &pc, active_vertex, ru, rv, zu, zv);
    double eta1 = gsum2(nx, ny, nz, periodic, ru, zu, rv, zv);
    if (eta1 != eta1) { status = ORC_ERR_NAN; break; }
    double beta = eta1 / eta0;
    for (size_t x = 0; x < nv; ++x) { du[x] = zu[x] + beta * du[x]; dv[x] = zv[x] + beta * dv[x]; }
    orc_halo_stag(nx, ny, nz, periodic, du);
    orc_halo_stag(nx, ny, nz, periodic, dv);
    orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, du, dv, qu, qv);
    eta0 = eta1;
    double eta2 = gsum2(nx, ny, nz, periodic, du, qu, dv, qv);
    double alpha = eta1 / eta2;
    if (alpha != alpha) { status = ORC_ERR_NAN; break; }
    for (size_t x = 0; x < nv; ++x) {
      xu[x] = xu[x] + alpha * du[x]; xv[x] = xv[x] + alpha * dv[x];
      ru[x] = ru[x] - alpha * qu[x]; rv[x] = rv[x] - alpha * qv[x];
    }
    if (n % ncheck == 0) {
      orc_halo_stag(nx, ny, nz, periodic, xu);
      orc_halo_stag(nx, ny, nz, periodic, xv);
      orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, xu, xv, zu, zv);
      for (size_t x = 0; x < nv; ++x) { ru[x] = bu[x] - zu[x]; rv[x] = bv[x] - zv[x]; }
      double L2_resid = sqrt(gsum2(nx, ny, nz, periodic, ru, ru, rv, rv));
      *err = L2_resid / L2_rhs;
      if (*err < tolerance) { *niters = n; status = ORC_OK; break; }
    }
  }
  free_precond(&pc);
  free(ru); free(rv); free(du); free(dv); free(qu); free(qv); free(zu); free(zv);
  return status;
}

/* pcg_solver_chrongear_3d (glissade_velo_higher_pcg.F90:965-1610). */
int orc_pcg_chrongear_3d(int nx, int ny, int nz, int periodic,
                         const int *active_vertex, const double *Auu,
                         const double *Auv, const double *Avu,
                         const double *Avv, const double *bu,
                         const double *bv, double *xu, double *xv,
                         int precond, int maxiters, double tolerance,
                         int ncheck, double *err, int *niters) {
  size_t nv = (size_t)nz * (nx - 1) * (ny - 1);
  double *ru = calloc(nv, 8), *rv = calloc(nv, 8), *du = calloc(nv, 8),
         *dv = calloc(nv, 8), *zu = calloc(nv, 8), *zv = calloc(nv, 8),
         *qu = calloc(nv, 8), *qv = calloc(nv, 8), *Azu = calloc(nv, 8),
         *Azv = calloc(nv, 8);
  precond_t pc;
  setup_precond(nx, ny, nz, precond, Auu, Avv, &pc);
  *niters = maxiters;
  *err = -1.0;
  double bb = gsum2(nx, ny, nz, periodic, bu, bu, bv, bv);
  double L2_rhs = sqrt(bb);
  orc_halo_stag(nx, ny, nz, periodic, xu);
  orc_halo_stag(nx, ny, nz, periodic, xv);
  orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, xu, xv, zu, zv);
  for (size_t x = 0; x < nv; ++x) { ru[x] = bu[x] - zu[x]; rv[x] = bv[x] - zv[x]; }
  orc_halo_stag(nx, ny, nz, periodic, ru);
  orc_halo_stag(nx, ny, nz, periodic, rv);
  apply_precond(nx, ny, nz, &pc, active_vertex, ru, rv, zu, zv);
  memcpy(du, zu, nv * 8); memcpy(dv, zv, nv * 8);
  orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, du, dv, qu, qv);
  double rho_old = gsum2(nx, ny, nz, periodic, ru, zu, rv, zv);
  double sigma = gsum2(nx, ny, nz, periodic, du, qu, dv, qv);
  orc_halo_stag(nx, ny, nz, periodic, qu);
  orc_halo_stag(nx, ny, nz, periodic, qv);
  double alpha = rho_old / sigma;
  int status = ORC_WARN_PCG_NOT_CONVERGED;
  if (alpha != alpha) status = ORC_ERR_NAN;
  else {
    for (size_t x = 0; x < nv; ++x) {
      xu[x] = xu[x] + alpha * du[x]; xv[x] = xv[x] + alpha * dv[x];
      ru[x] = ru[x] - alpha * qu[x]; rv[x] = rv[x] - alpha * qv[x];
    }
    for (int n = 2; n <= maxiters; ++n) {
      apply_precond(nx, ny, nz, &pc, active_vertex, ru, rv, zu, zv);
      orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, zu, zv, Azu, Azv);
      double rho = gsum2(nx, ny, nz, periodic, ru, zu, rv, zv);
      double delta = gsum2(nx, ny, nz, periodic, Azu, zu, Azv, zv);
      orc_halo_stag(nx, ny, nz, periodic, Azu);
      orc_halo_stag(nx, ny, nz, periodic, Azv);
      double beta = rho / rho_old;
      sigma = delta - beta * rho / alpha;
      alpha = rho / sigma;
      rho_old = rho;
      if (alpha != alpha) { status = ORC_ERR_NAN; break; }
      for (size_t x = 0; x < nv; ++x) {
        du[x] = zu[x] + beta * du[x]; dv[x] = zv[x] + beta * dv[x];
        qu[x] = Azu[x] + beta * qu[x]; qv[x] = Azv[x] + beta * qv[x];
        xu[x] = xu[x] + alpha * du[x]; xv[x] = xv[x] + alpha * dv[x];
        ru[x] = ru[x] - alpha * qu[x]; rv[x] = rv[x] - alpha * qv[x];
      }
      if (n % ncheck == 0) {
        orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, xu, xv, zu, zv);
        for (size_t x = 0; x < nv; ++x) { ru[x] = bu[x] - zu[x]; rv[x] = bv[x] - zv[x]; }
        double rr = gsum2(nx, ny, nz, periodic, ru, ru, rv, rv);
        *err = sqrt(rr) / L2_rhs;
        if (*err < tolerance) { *niters = n; status = ORC_OK; break; }
        orc_halo_stag(nx, ny, nz, periodic, ru);
        orc_halo_stag(nx, ny, nz, periodic, rv);
      }
    }
  }
  free_precond(&pc);
  free(ru); free(rv); free(du); free(dv); free(zu); free(zv); free(qu);
  free(qv); free(Azu); free(Azv);
  return status;
}

/* compute_residual_vector_3d (:8768-8927). */
static void residual_vector_3d(int nx, int ny, int nz, int periodic,
                               const int *active_vertex, const double *Auu,
                               const double *Auv, const double *Avu,
                               const double *Avv, const double *bu,
                               const double *bv, const double *uvel,
                               const double *vvel, double *L2_norm,
                               double *L2_rel) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  size_t nv = (size_t)nz * (nx - 1) * (ny - 1);
  double *resu = calloc(nv, 8), *resv = calloc(nv, 8);
  orc_matvec_3d(nx, ny, nz, periodic, active_vertex, Auu, Auv, Avu, Avv, uvel, vvel, resu, resv);
  double L2 = 0.0, L2b = 0.0;
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      for (int k = 1; k <= nz; ++k) {
        size_t x = IX(k, i, j);
        resu[x] = resu[x] - bu[x];
        resv[x] = resv[x] - bv[x];
        L2 = L2 + resu[x] * resu[x] + resv[x] * resv[x];
      }
    }
  *L2_norm = sqrt(L2);
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i) {
      if (!active_vertex[IV(i, j)]) continue;
      for (int k = 1; k <= nz; ++k) {
        size_t x = IX(k, i, j);
        L2b = L2b + bu[x] * bu[x] + bv[x] * bv[x];
      }
    }
  L2b = sqrt(L2b);
  *L2_rel = L2b > 0.0 ? *L2_norm / L2b : 0.0;
  free(resu);
  free(resv);
}

/* compute_residual_velocity_3d (:9111-9234). */
static double residual_velocity_3d(int nx, int ny, int nz, int periodic,
                                   int whichresid, const double *uvel,
                                   const double *vvel, const double *usav,
                                   const double *vsav) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  double r = 0.0;
  long count = 0;
  int kmax = (whichresid == ORC_RESID_MAXU_NO_UBAS || whichresid == ORC_RESID_MEANU) ? nz - 1 : nz;
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i)
      for (int k = 1; k <= kmax; ++k) {
        size_t x = IX(k, i, j);
        double speed = sqrt(uvel[x] * uvel[x] + vvel[x] * vvel[x]);
        if (speed != 0.0) {
          double oldspeed = sqrt(usav[x] * usav[x] + vsav[x] * vsav[x]);
          double diff = fabs((oldspeed - speed) / speed);
          if (whichresid == ORC_RESID_MEANU) { r = r + diff; ++count; }
          else if (diff > r) r = diff;
        }
      }
  if (whichresid == ORC_RESID_MEANU && count > 0) r = r / (double)count;
  return r;
}

/* load_vector_gravity (:4317-4532). */
static void load_vector_gravity(const orc_model *m, const orc_setup *s) {
  const int nx = m->nx, ny = m->ny, nz = m->nz, nhalo = m->nhalo;
  const double vol0 = 1.0e9, rhoi = m->rhoi, grav = m->grav;
  const double dx = m->dx, dy = m->dy;
  if (m->which_assemble_taud == ORC_ASSEMBLE_LOCAL) {
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        if (!s->active_vertex[IV(i, j)]) continue;
        for (int k = 1; k <= nz; ++k) {
          double dz = s->stagthck[IV(i, j)] * (s->stagwbndsigma[k] - s->stagwbndsigma[k - 1]);
          s->loadu[IX(k, i, j)] = s->loadu[IX(k, i, j)] - rhoi * grav * dx * dy * dz / vol0 * s->dusrf_dx[IV(i, j)];
          s->loadv[IX(k, i, j)] = s->loadv[IX(k, i, j)] - rhoi * grav * dx * dy * dz / vol0 * s->dusrf_dy[IV(i, j)];
        }
      }
    return;
  }
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!s->active_cell[IC(i, j)]) continue;
      for (int k = 1; k <= nz - 1; ++k) {
        double x[8], y[8], z[8], dsdx[8], dsdy[8];
        for (int n = 0; n < 8; ++n) {
          int in = i + ishift[6][n], jn = j + jshift[6][n], kn = k + kshift[6][n];
          x[n] = s->xVertex[IV(in, jn)];
          y[n] = s->yVertex[IV(in, jn)];
          z[n] = s->stagusrf[IV(in, jn)] - s->sigma[kn - 1] * s->stagthck[IV(in, jn)];
          dsdx[n] = s->dusrf_dx[IV(in, jn)];
          dsdy[n] = s->dusrf_dy[IV(in, jn)];
        }
        for (int p = 0; p < 8; ++p) {
          double ddx[8], ddy[8], ddz[8], detJ;
          basis_derivs_3d(x, y, z, p, ddx, ddy, ddz, &detJ);
          double sx = 0.0, sy = 0.0;
          for (int n = 0; n < 8; ++n) { sx = sx + phi3[n][p] * dsdx[n]; sy = sy + phi3[n][p] * dsdy[n]; }
          for (int n = 0; n < 8; ++n) {
            int in = i + ishift[6][n], jn = j + jshift[6][n], kn = k + kshift[6][n];
            s->loadu[IX(kn, in, jn)] = s->loadu[IX(kn, in, jn)] - rhoi * grav * wqp[p] * detJ / vol0 * sx * phi3[n][p];
            s->loadv[IX(kn, in, jn)] = s->loadv[IX(kn, in, jn)] - rhoi * grav * wqp[p] * detJ / vol0 * sy * phi3[n][p];
          }
        }
      }
    }
}

/* lateral_shelf_bc (:4659-4950). face: 0 west, 1 east, 2 south, 3 north. */
static void lateral_shelf_bc(const orc_model *m, const orc_setup *s, int face,
                             int iCell, int jCell) {
  const int nx = m->nx, nz = m->nz;
  const double vol0 = 1.0e9, rhoi = m->rhoi, rhoo = m->rhoo, grav = m->grav;
  int iN[4], jN[4], kN[4];
  double x[4], y[4], sv[4], h[4];
  if (face == 0) { iN[0] = iCell - 1; jN[0] = jCell; iN[1] = iCell - 1; jN[1] = jCell - 1; }
  else if (face == 1) { iN[0] = iCell; jN[0] = jCell - 1; iN[1] = iCell; jN[1] = jCell; }
  else if (face == 2) { iN[0] = iCell - 1; jN[0] = jCell - 1; iN[1] = iCell; jN[1] = jCell - 1; }
  else { iN[0] = iCell; jN[0] = jCell; iN[1] = iCell - 1; jN[1] = jCell; }
  const double *coord = (face <= 1) ? s->yVertex : s->xVertex;
  x[0] = coord[IV(iN[0], jN[0])];
  x[1] = coord[IV(iN[1], jN[1])];
  iN[2] = iN[1]; jN[2] = jN[1]; iN[3] = iN[0]; jN[3] = jN[0];
  x[2] = x[1]; x[3] = x[0];
  sv[0] = s->stagusrf[IV(iN[0], jN[0])]; sv[1] = s->stagusrf[IV(iN[1], jN[1])];
  sv[2] = sv[1]; sv[3] = sv[0];
  h[0] = s->stagthck[IV(iN[0], jN[0])]; h[1] = s->stagthck[IV(iN[1], jN[1])];
  h[2] = h[1]; h[3] = h[0];
  for (int k = 1; k <= nz - 1; ++k) {
    y[0] = sv[0] - s->sigma[k] * h[0];
    y[1] = sv[1] - s->sigma[k] * h[1];
    y[2] = sv[2] - s->sigma[k - 1] * h[2];
    y[3] = sv[3] - s->sigma[k - 1] * h[3];
    kN[0] = k + 1; kN[1] = k + 1; kN[2] = k; kN[3] = k;
    for (int p = 0; p < 4; ++p) {
      double detJ;
      basis_detJ_2d(x, y, p, &detJ);
      detJ = fabs(detJ);
      double hq = 0.0, sq = 0.0;
      for (int n = 0; n < 4; ++n) { hq = hq + phi2[n][p] * h[n]; sq = sq + phi2[n][p] * sv[n]; }
      double t = 1.0 - fmin(sq / hq, 1.0);
      double p_av = 0.5 * rhoi * grav * hq - 0.5 * rhoo * grav * hq * (t * t);
      for (int n = 0; n < 4; ++n) {
        size_t xidx = IX(kN[n], iN[n], jN[n]);
        double f = p_av * wqp2[p] * detJ / vol0 * phi2[n][p];
        if (face == 0) s->loadu[xidx] = s->loadu[xidx] - f;
        else if (face == 1) s->loadu[xidx] = s->loadu[xidx] + f;
        else if (face == 2) s->loadv[xidx] = s->loadv[xidx] - f;
        else s->loadv[xidx] = s->loadv[xidx] + f;
      }
    }
  }
}

/* load_vector_lateral_bc (:4536-4655); calving_front_mask = 0. */
static void load_vector_lateral_bc(const orc_model *m, const orc_setup *s) {
  const int nx = m->nx, ny = m->ny, nhalo = m->nhalo;
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!s->active_cell[IC(i, j)]) continue;
      if (s->ocean_mask[IC(i - 1, j)] == 1) lateral_shelf_bc(m, s, 0, i, j);
      if (s->ocean_mask[IC(i + 1, j)] == 1) lateral_shelf_bc(m, s, 1, i, j);
      if (s->ocean_mask[IC(i, j - 1)] == 1) lateral_shelf_bc(m, s, 2, i, j);
      if (s->ocean_mask[IC(i, j + 1)] == 1) lateral_shelf_bc(m, s, 3, i, j);
    }
}

/* Setup part of glissade_velo_higher_solve (:1270-2199) plus the masks and
 * grounded fraction computed by glissade_diagnostic_variable_solve
 * (glissade.F90:1818-1846). */
int orc_setup_solve(const orc_model *m, orc_setup *s, double *uvel,
                    double *vvel) {
  init_tables();
  const int nx = m->nx, ny = m->ny, nz = m->nz, nhalo = m->nhalo;
  if (nhalo != 2 || nx < 6 || ny < 6 || nz < 2) return ORC_ERR_ARGS;
  size_t nc = (size_t)nx * ny, nvx = (size_t)(nx - 1) * (ny - 1), n3 = nvx * nz;
  orc_sigma_glide(nz, s->sigma, s->stagwbndsigma);
  memset(s->umask_dirichlet, 0, n3 * sizeof(int));
  memset(s->vmask_dirichlet, 0, n3 * sizeof(int));
  if (m->which_babc == ORC_BABC_NO_SLIP)
    for (size_t v = 0; v < nvx; ++v) {
      s->umask_dirichlet[v * nz + (nz - 1)] = 1;
      s->vmask_dirichlet[v * nz + (nz - 1)] = 1;
    }
  if (m->kinbcmask)
    for (size_t v = 0; v < nvx; ++v)
      if (m->kinbcmask[v] == 1)
        for (int k = 0; k < nz; ++k) {
          s->umask_dirichlet[v * nz + k] = 1;
          s->vmask_dirichlet[v * nz + k] = 1;
        }
  int *active_ice = malloc(nc * sizeof(int));
  int *ipl = malloc(nc * sizeof(int));
  orc_get_masks(nx, ny, m->periodic, m->thck, m->topg, m->eus, m->thklim,
                m->rhoi, m->rhoo, s->ice_mask, s->floating_mask,
                s->ocean_mask, s->land_mask, active_ice);
  for (size_t c = 0; c < nc; ++c)
    ipl[c] = (active_ice[c] == 1 || s->land_mask[c] == 1) ? 1 : 0;
  orc_stagger(nx, ny, m->thck, s->stagthck, ipl, 1);
  orc_stagger(nx, ny, m->usrf, s->stagusrf, ipl, 1);
  orc_surface_gradient(nx, ny, m->periodic, m->dx, m->dy, active_ice,
                       s->land_mask, m->usrf, m->thck, m->thklim,
                       m->thck_gradient_ramp, m->which_gradient,
                       m->which_gradient_margin, m->max_slope, s->dusrf_dx,
                       s->dusrf_dy);
  /* get_vertex_geometry (:4163-4313) */
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      s->xVertex[IV(i, j)] = m->dx * i;
      s->yVertex[IV(i, j)] = m->dy * j;
    }
  memset(s->active_cell, 0, nc * sizeof(int));
  memset(s->active_vertex, 0, nvx * sizeof(int));
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i)
      if (active_ice[IC(i, j)] == 1) s->active_cell[IC(i, j)] = 1;
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i)
      if (s->active_cell[IC(i, j)]) {
        s->active_vertex[IV(i - 1, j - 1)] = 1; s->active_vertex[IV(i, j - 1)] = 1;
        s->active_vertex[IV(i - 1, j)] = 1; s->active_vertex[IV(i, j)] = 1;
      }
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, m->periodic, &ilo, &ihi, &jlo, &jhi);
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i)
      if (!s->active_vertex[IV(i, j)])
        for (int k = 1; k <= nz; ++k) { uvel[IX(k, i, j)] = 0.0; vvel[IX(k, i, j)] = 0.0; }
  /* flwafact (:1919-1939) */
  memset(s->flwafact, 0, (size_t)(nz - 1) * nc * sizeof(double));
  for (int j = 1 + nhalo; j <= ny - nhalo + 1; ++j)
    for (int i = 1 + nhalo; i <= nx - nhalo + 1; ++i)
      for (int k = 1; k <= nz - 1; ++k)
        if (m->flwa[IFL(k, i, j)] > 0.0)
          s->flwafact[IFL(k, i, j)] = 0.5 * pow(m->flwa[IFL(k, i, j)], -1.0 / 3.0);
  memset(s->loadu, 0, n3 * sizeof(double));
  memset(s->loadv, 0, n3 * sizeof(double));
  load_vector_gravity(m, s);
  load_vector_lateral_bc(m, s);
  orc_grounded_fraction(nx, ny, s->ice_mask, s->floating_mask, s->land_mask,
                        m->which_ground, s->f_ground);
  free(active_ice);
  free(ipl);
  return ORC_OK;
}

/* calcbeta (glissade_basal_traction.F90:67-598) as called at the start of
 * each Picard iteration (glissade_velo_higher.F90:2502-2517) with ubas,
 * vbas = uvel(nz,:,:), vvel(nz,:,:) (:2241-2242): the speed with its
 * 0.01 m/a floor (:181) and optional cap (:187-189); the law; beta *
 * f_ground (:540); the grounded minimum (:560-566); the validity check
 * (:570-582); the halo update.  gn = 3 is an integer in the reference
 * (glimmer_physcon.F90:75): N**gn is a product, 1/gn a real division. */
int orc_calcbeta(const orc_model *m, const orc_setup *s, const double *uvel,
                 const double *vvel, double *beta_internal) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const orc_basal_physics *bp = m->basal;
  const double smallnum = 1.0e-2, pi = 3.14159265358979;
  double *flwa_basal_stag = NULL;
  if (m->which_babc == ORC_BABC_COULOMB_FRICTION) {
    /* basal-layer flwa staggered over cells with thck > 0 (:393-398) */
    int *imask = calloc((size_t)nx * ny, sizeof(int));
    double *flwa_basal = calloc((size_t)nx * ny, sizeof(double));
    flwa_basal_stag = calloc((size_t)(nx - 1) * (ny - 1), sizeof(double));
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        imask[IC(i, j)] = m->thck[IC(i, j)] > 0.0 ? 1 : 0;
        flwa_basal[IC(i, j)] = m->flwa[IFL(nz - 1, i, j)];
      }
    orc_stagger(nx, ny, flwa_basal, flwa_basal_stag, imask, 1);
    free(imask);
    free(flwa_basal);
  }
  int status = ORC_OK;
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const size_t v = IV(i, j);
      const double ub = uvel[IX(nz, i, j)], vb = vvel[IX(nz, i, j)];
      double speed = sqrt(ub * ub + vb * vb + smallnum * smallnum);
      double b = 0.0;
      if (bp && bp->beta_powerlaw_umax > 0.0 && bp->beta_powerlaw_umax < speed)
        speed = bp->beta_powerlaw_umax;
      switch (m->which_babc) {
        case ORC_BABC_BETA_CONSTANT:
          b = m->beta_const;
          break;
        case ORC_BABC_BETA_EXTERNAL:
          b = m->beta_external[v];
          break;
        case ORC_BABC_PSEUDO_PLASTIC: { /* :207-264 */
          const double bed = m->topg[IC(i, j)] - m->eus;
          double phi;
          if (bed <= bp->pseudo_plastic_bedmin) phi = bp->pseudo_plastic_phimin;
          else if (bed >= bp->pseudo_plastic_bedmax) phi = bp->pseudo_plastic_phimax;
          else phi = bp->pseudo_plastic_phimin +
                     ((bed - bp->pseudo_plastic_bedmin) /
                      (bp->pseudo_plastic_bedmax - bp->pseudo_plastic_bedmin)) *
                         (bp->pseudo_plastic_phimax - bp->pseudo_plastic_phimin);
          const double tanphi = tan(phi * pi / 180.0);
          const double tau_c = tanphi * bp->effecpress_stag[v];
          b = tau_c / (pow(bp->pseudo_plastic_u0, bp->pseudo_plastic_q) *
                       pow(speed, 1.0 - bp->pseudo_plastic_q));
          break;
        }
        case ORC_BABC_YIELD_PICARD: /* :266-277 */
          b = bp->mintauf_tau0[v] / sqrt(ub * ub + vb * vb + smallnum * smallnum);
          break;
        case ORC_BABC_POWERLAW: /* :357-363 */
          b = bp->powerlaw_c * pow(speed, 1.0 / bp->powerlaw_m - 1.0);
          break;
        case ORC_BABC_POWERLAW_EFFECPRESS: { /* :365-382, p = 3, q = 1 */
          const double p = 3.0, q = 1.0;
          b = pow(bp->friction_powerlaw_k, -1.0 / p) * pow(bp->effecpress_stag[v], q / p) *
              pow(speed, 1.0 / p - 1.0);
          break;
        }
        case ORC_BABC_COULOMB_FRICTION: { /* :384-424 */
          const double N = bp->effecpress_stag[v];
          const double cs = bp->c_space_factor_stag ? bp->c_space_factor_stag[v] : 1.0;
          const double big_lambda = (bp->coulomb_bump_wavelength / bp->coulomb_bump_max_slope) *
                                    flwa_basal_stag[v];
          b = bp->coulomb_c * cs * N * pow(speed, 1.0 / 3 - 1.0) *
              pow(speed + N * N * N * big_lambda, -1.0 / 3);
          if (b > 1.0e8) b = 1.0e8;
          break;
        }
        case ORC_BABC_COULOMB_POWERLAW_SCHOOF: { /* :426-470 */
          const double N = bp->effecpress_stag[v], mm = bp->powerlaw_m;
          const double numerator = bp->powerlaw_c * bp->coulomb_c * N;
          const double denominator = pow(pow(bp->powerlaw_c, mm) * speed + pow(bp->coulomb_c * N, mm),
                                         1.0 / mm);
          b = (numerator / denominator) * pow(speed, 1.0 / mm - 1.0);
          if (b > 1.0e8) b = 1.0e8;
          break;
        }
        case ORC_BABC_COULOMB_POWERLAW_TSAI: { /* :472-509 */
          const double taub_powerlaw = bp->powerlaw_c * pow(speed, 1.0 / bp->powerlaw_m);
          const double taub_coulomb = bp->coulomb_c * bp->effecpress_stag[v];
          b = (taub_coulomb <= taub_powerlaw) ? taub_coulomb / speed : taub_powerlaw / speed;
          break;
        }
        default:
          b = 0.0;
          break;
      }
      b = b * s->f_ground[v];
      if (s->f_ground[v] > 0.0 && b < m->beta_grounded_min) b = m->beta_grounded_min;
      if (!(b >= 0.0)) status = ORC_ERR_BAD_BETA;
      beta_internal[v] = b;
    }
  free(flwa_basal_stag);
  if (status != ORC_OK) return status;
  orc_halo_stag(nx, ny, 1, m->periodic, beta_internal);
  return ORC_OK;
}

int orc_assemble_system(const orc_model *m, const orc_setup *s,
                        const double *beta_internal, const double *uvel,
                        const double *vvel, double *efvs, double *Auu,
                        double *Auv, double *Avu, double *Avv, double *bu,
                        double *bv, long *nNonzeros) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  size_t n3 = (size_t)nz * (nx - 1) * (ny - 1);
  int st = orc_assemble_3d(nx, ny, nz, m->nhalo, s->sigma, s->active_cell,
                           s->xVertex, s->yVertex, uvel, vvel, s->stagusrf,
                           s->stagthck, s->flwafact, m->which_efvs,
                           m->efvs_constant, efvs, Auu, Auv, Avu, Avv);
  if (st != ORC_OK) return st;
  if (m->which_babc != ORC_BABC_NO_SLIP)
    basal_sliding_bc(nx, ny, nz, m->nhalo, m->dx, m->dy, s->active_cell,
                     s->active_vertex, beta_internal, s->xVertex, s->yVertex,
                     m->which_assemble_beta, Auu, Avv);
  memcpy(bu, s->loadu, n3 * sizeof(double));
  memcpy(bv, s->loadv, n3 * sizeof(double));
  dirichlet_bc_3d(nx, ny, nz, m->nhalo, s->active_vertex, s->umask_dirichlet,
                  s->vmask_dirichlet, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv);
  orc_halo_stag(nx, ny, 27 * nz, m->periodic, Auu);
  orc_halo_stag(nx, ny, 27 * nz, m->periodic, Auv);
  orc_halo_stag(nx, ny, 27 * nz, m->periodic, Avu);
  orc_halo_stag(nx, ny, 27 * nz, m->periodic, Avv);
  orc_halo_stag(nx, ny, nz, m->periodic, bu);
  orc_halo_stag(nx, ny, nz, m->periodic, bv);
  check_symmetry_assembled_3d(nx, ny, nz, m->periodic, s->active_vertex, Auu,
                              Auv, Avu, Avv);
  *nNonzeros = count_nonzeros_3d(nx, ny, nz, m->periodic, s->active_vertex,
                                 Auu, Auv, Avu, Avv);
  return ORC_OK;
}

static void *xalloc(size_t n) { return calloc(n ? n : 1, 1); }

void orc_setup_alloc(const orc_model *m, orc_setup *s) {
  size_t nx = m->nx, ny = m->ny, nz = m->nz;
  size_t nc = nx * ny, nvx = (nx - 1) * (ny - 1), n3 = nvx * nz;
  s->sigma = xalloc(nz * 8); s->stagwbndsigma = xalloc((nz + 1) * 8);
  s->stagusrf = xalloc(nvx * 8); s->stagthck = xalloc(nvx * 8);
  s->dusrf_dx = xalloc(nvx * 8); s->dusrf_dy = xalloc(nvx * 8);
  s->xVertex = xalloc(nvx * 8); s->yVertex = xalloc(nvx * 8);
  s->f_ground = xalloc(nvx * 8); s->flwafact = xalloc((nz - 1) * nc * 8);
  s->loadu = xalloc(n3 * 8); s->loadv = xalloc(n3 * 8);
  s->active_cell = xalloc(nc * 4); s->active_vertex = xalloc(nvx * 4);
  s->umask_dirichlet = xalloc(n3 * 4); s->vmask_dirichlet = xalloc(n3 * 4);
  s->ice_mask = xalloc(nc * 4); s->floating_mask = xalloc(nc * 4);
  s->ocean_mask = xalloc(nc * 4); s->land_mask = xalloc(nc * 4);
}

void orc_setup_free(orc_setup *s) {
  free(s->sigma); free(s->stagwbndsigma); free(s->stagusrf); free(s->stagthck);
  free(s->dusrf_dx); free(s->dusrf_dy); free(s->xVertex); free(s->yVertex);
  free(s->f_ground); free(s->flwafact); free(s->loadu); free(s->loadv);
  free(s->active_cell); free(s->active_vertex); free(s->umask_dirichlet);
  free(s->vmask_dirichlet); free(s->ice_mask); free(s->floating_mask);
  free(s->ocean_mask); free(s->land_mask);
}

/* ---------------------------------------------------------------------
 * Shallow-shelf (SSA) branch of glissade_velo_higher_solve: the 2-D
 * solve (solve_2d, :1125-1128) for whichapprox = HO_APPROX_SSA.  The 2-D
 * matrix (indxA_2d, 9 entries) is kept in the kA = 0 slice of the 27-entry
 * layout with nz = 1; the 2-D matvec, PCG, Dirichlet, symmetry and
 * nonzero-count routines of the reference are the 3-D ones at nz = 1 with
 * the same loop orders (matvec_multiply_structured_2d :2651-2755 against
 * _3d :2533-2647; pcg_solver_standard_2d :553-961 and chrongear_2d
 * :1614-2146 against their 3-D forms; dirichlet_boundary_conditions_2d
 * :8582-8764), so those are called with nz = 1.
 * ------------------------------------------------------------------- */

/* get_basis_function_derivatives_2d (:6583-6751) with the reference
 * element's derivatives dxr, dyr at one point (a quadrature point, or the
 * element centre, :589-597). */
static int basis_derivs_2d_at(const double *x, const double *y, const double *dxr,
                              const double *dyr, double *dx, double *dy, double *detJ) {
  double J11 = 0.0, J12 = 0.0, J21 = 0.0, J22 = 0.0;
  for (int n = 0; n < 4; ++n) {
    J11 = J11 + dxr[n] * x[n];
    J12 = J12 + dxr[n] * y[n];
    J21 = J21 + dyr[n] * x[n];
    J22 = J22 + dyr[n] * y[n];
  }
  const double d = J11 * J22 - J12 * J21;
  *detJ = d;
  if (!(fabs(d) > 0.0)) return ORC_ERR_SINGULAR_JAC;
  const double i11 = J22 / d, i12 = -J12 / d, i21 = -J21 / d, i22 = J11 / d;
  for (int n = 0; n < 4; ++n) {
    dx[n] = i11 * dxr[n] + i12 * dyr[n];
    dy[n] = i21 * dxr[n] + i22 * dyr[n];
  }
  return ORC_OK;
}

static int basis_derivs_2d(const double *x, const double *y, int p, double *dx,
                           double *dy, double *detJ) {
  double dxr[4], dyr[4];
  for (int n = 0; n < 4; ++n) { dxr[n] = dxr2[n][p]; dyr[n] = dyr2[n][p]; }
  return basis_derivs_2d_at(x, y, dxr, dyr, dx, dy, detJ);
}

/* compute_effective_viscosity, SSA branch (:7199-7378) with the vertically
 * averaged flow factor. */
static double effective_viscosity_ssa(int whichefvs, double efvs_constant,
                                      const double *dx, const double *dy,
                                      const double *u, const double *v,
                                      double flwafact) {
  const double effstrain_min = 1.0e-8;
  const double p_effstr = (1.0 - 3.0) / 3.0;
  const double p2_effstr = p_effstr / 2.0;
  if (whichefvs == ORC_EFVS_CONSTANT) return efvs_constant;
  if (whichefvs == ORC_EFVS_FLOWFACT) {
    const double scyr = 31536000.0;
    double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    return flwafact * pow(effstrain, p_effstr);
  }
  double ux = 0, uy = 0, vx = 0, vy = 0;
  for (int n = 0; n < 4; ++n) {
    ux = ux + dx[n] * u[n];
    uy = uy + dy[n] * u[n];
    vx = vx + dx[n] * v[n];
    vy = vy + dy[n] * v[n];
  }
  double sq = effstrain_min * effstrain_min +
              (ux * ux + vy * vy + ux * vy + 0.25 * ((vx + uy) * (vx + uy)));
  return flwafact * pow(sq, p2_effstr);
}

/* compute_effective_viscosity_L1L2 (:7382-7618): the viscosity of each
 * layer k = 1..nz-1 at one quadrature point (phi, dx, dy its basis values
 * and derivatives; u, v, h, dsdx, dsdy the corner values).  With Glen's
 * law (n = 3) tau_parallel solves x^3 + a x + b = 0, a = tau_perp^2 =
 * (rhoi grav (h sigma(k+1)) |grad s|)^2, b = -effstrain / A, by Cardano's
 * formula: x = (-b/2 + c)^(1/3) - (b/2 + c)^(1/3), c = sqrt(b^2/4 +
 * a^3/27), the second root in its first-order form -a / (3 |b|^(1/3))
 * when a^3/27 <= 1e-6 b^2/4; then efvs = 1 / (2 A (x^2 + tau_perp^2)). */
static void effective_viscosity_l1l2(int whichefvs, double efvs_constant, int nz,
                                     const double *sigma, int p, const double *dx,
                                     const double *dy, const double *u, const double *v,
                                     const double *h, const double *dsdx, const double *dsdy,
                                     const double *flwa, const double *flwafact, double rhoi,
                                     double grav, double *efvs) {
  const double effstrain_min = 1.0e-8;
  const double p_effstr = (1.0 - 3.0) / 3.0;
  if (whichefvs == ORC_EFVS_CONSTANT) {
    for (int k = 0; k < nz - 1; ++k) efvs[k] = efvs_constant;
    return;
  }
  if (whichefvs == ORC_EFVS_FLOWFACT) {
    const double scyr = 31536000.0;
    const double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    for (int k = 0; k < nz - 1; ++k) efvs[k] = flwafact[k] * pow(effstrain, p_effstr);
    return;
  }
  double ux = 0.0, uy = 0.0, vx = 0.0, vy = 0.0, sx = 0.0, sy = 0.0, thck = 0.0;
  for (int n = 0; n < 4; ++n) {
    ux = ux + dx[n] * u[n];
    uy = uy + dy[n] * u[n];
    vx = vx + dx[n] * v[n];
    vy = vy + dy[n] * v[n];
    sx = sx + phi2[n][p] * dsdx[n];
    sy = sy + phi2[n][p] * dsdy[n];
    thck = thck + phi2[n][p] * h[n];
  }
  const double effstrainsq = effstrain_min * effstrain_min + ux * ux + vy * vy + ux * vy +
                             0.25 * ((vx + uy) * (vx + uy));
  const double effstrain = sqrt(effstrainsq);
  for (int k = 1; k <= nz - 1; ++k) {
    const double depth = thck * sigma[k];
    const double grads = sqrt(sx * sx + sy * sy);
    const double tau_perp = rhoi * grav * depth * grads;
    const double a = tau_perp * tau_perp;
    const double b = -effstrain / flwa[k - 1];
    const double c = sqrt(b * b / 4.0 + a * a * a / 27.0);
    const double rootA = pow(-b / 2.0 + c, 1.0 / 3.0);
    double rootB;
    if (a * a * a / 27.0 > 1.0e-6 * (b * b / 4.0))
      rootB = -pow(b / 2.0 + c, 1.0 / 3.0);
    else
      rootB = -a / (3.0 * pow(fabs(b), 1.0 / 3.0));
    const double tau_parallel = rootA + rootB;
    efvs[k - 1] = 1.0 / (2.0 * flwa[k - 1] * (tau_parallel * tau_parallel + tau_perp * tau_perp));
  }
}

/* compute_effective_viscosity_diva (:7622-7864), the default non-cubic
 * form: the viscosity of each layer k at one quadrature point from the
 * horizontal strain rates of the mean velocity and the vertical shear
 * (du/dz, dv/dz) = tau_b stagsigma(k) / efvs_old(k), tau_b the basal
 * traction interpolated to the point; efvs (in: the last assembly's
 * value, 0 = none yet, then the value at the 1e-8 /a strain-rate floor;
 * out: the new value). */
static void effective_viscosity_diva(int whichefvs, double efvs_constant, int nz,
                                     const double *sigma, int p, const double *dx,
                                     const double *dy, const double *u, const double *v,
                                     const double *bx, const double *by,
                                     const double *flwafact, double *efvs) {
  const double effstrain_min = 1.0e-8;
  const double p_effstr = (1.0 - 3.0) / 3.0;
  const double p2_effstr = p_effstr / 2;
  if (whichefvs == ORC_EFVS_CONSTANT) {
    for (int k = 0; k < nz - 1; ++k) efvs[k] = efvs_constant;
    return;
  }
  if (whichefvs == ORC_EFVS_FLOWFACT) {
    const double scyr = 31536000.0;
    const double effstrain = (500.0 / scyr) / 200.0e3 * scyr;
    for (int k = 0; k < nz - 1; ++k) efvs[k] = flwafact[k] * pow(effstrain, p_effstr);
    return;
  }
  double ux = 0.0, uy = 0.0, vx = 0.0, vy = 0.0, taux = 0.0, tauy = 0.0;
  for (int n = 0; n < 4; ++n) {
    ux = ux + dx[n] * u[n];
    uy = uy + dy[n] * u[n];
    vx = vx + dx[n] * v[n];
    vy = vy + dy[n] * v[n];
    taux = taux + phi2[n][p] * bx[n];
    tauy = tauy + phi2[n][p] * by[n];
  }
  for (int k = 1; k <= nz - 1; ++k) {
    if (efvs[k - 1] == 0.0) efvs[k - 1] = flwafact[k - 1] * pow(effstrain_min, p_effstr);
    const double stagsigma = (sigma[k - 1] + sigma[k]) / 2.0;
    const double du_dz = taux * stagsigma / efvs[k - 1];
    const double dv_dz = tauy * stagsigma / efvs[k - 1];
    const double effstrainsq = effstrain_min * effstrain_min + ux * ux + vy * vy + ux * vy +
                               0.25 * ((vx + uy) * (vx + uy)) + 0.25 * (du_dz * du_dz + dv_dz * dv_dz);
    efvs[k - 1] = flwafact[k - 1] * pow(effstrainsq, p2_effstr);
  }
}

/* compute_integrals_diva (:5601-5726): per quadrature point the integral
 * of depth / efvs from the bed up to each level, averaged over the points
 * (omega_k, Goldberg 2011 eq. 32, over H), and its layer-midpoint integral
 * over the column (omega, eq. 35 over H).  eq holds the cell's point
 * viscosities [p][k]. */
static void integrals_diva(int nz, const double *sigma, double thck, const double *eq,
                           double *omega_k, double *omega) {
  double okp[4][65];
  for (int p = 0; p < 4; ++p) {
    okp[p][nz - 1] = 0.0;
    for (int k = nz - 1; k >= 1; --k) {  /* layer k between levels k and k+1 (1-based) */
      const double depth = 0.5 * (sigma[k - 1] + sigma[k]);
      const double dz = (sigma[k] - sigma[k - 1]) * thck;
      okp[p][k - 1] = okp[p][k] + depth / eq[(size_t)p * (nz - 1) + (k - 1)] * dz;
    }
  }
  for (int k = 0; k < nz; ++k) {
    double s = 0.0;
    for (int p = 0; p < 4; ++p) s = s + okp[p][k];
    omega_k[k] = s / 4;
  }
  double om = 0.0;
  for (int k = 1; k <= nz - 1; ++k) {
    const double layer_avg = 0.5 * (omega_k[k - 1] + omega_k[k]);
    const double dz = sigma[k] - sigma[k - 1];
    om = om + layer_avg * dz;
  }
  *omega = om;
}

/* DIVA state of one 2-D assembly: the viscosity of each layer at each
 * point efvs_qp_3d (in: the last assembly's, out: this one's), the basal
 * traction at the vertices, the cell thickness, and the integrals the
 * assembly produces. */
typedef struct {
  double *eq3;                   /* (nz-1,4,nx,ny) */
  const double *btx, *bty;       /* (nx-1,ny-1) */
  const double *thck;            /* (nx,ny) */
  double *omega_k;               /* (nz,nx,ny) */
  double *omega;                 /* (nx,ny) */
} diva_state;

/* assemble_stiffness_matrix_2d (:5208-5595), SSA and L1L2 branches: per
 * active cell, 2x2 Gauss points; the SSA efvs from the vertically averaged
 * flow factor (glissade_vertical_average, glissade_grid_operators.F90:
 * 1172-1236), the L1L2 efvs of each layer (effective_viscosity_l1l2)
 * averaged over the column with the weights sigma(k+1) - sigma(k); the
 * element matrix with h efvs (compute_element_matrix :7868-7986), scatter
 * by element_to_global_matrix_2d (:8058-8121); efvs(k,i,j) = the mean of
 * the point values of layer k (SSA: the one value on every layer). */
static int assemble_2d(int approx, int nx, int ny, int nz, int nhalo, const double *sigma,
                       const int *active_cell, const double *xVertex,
                       const double *yVertex, const double *u2, const double *v2,
                       const double *stagthck, const double *flwafact, const double *flwa,
                       const double *dusrf_dx, const double *dusrf_dy, double rhoi,
                       double grav, const diva_state *dv, int whichefvs,
                       double efvs_constant, double *efvs, double *Auu, double *Auv,
                       double *Avu, double *Avv) {
  init_tables();
  const double vol0 = 1.0e9;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1);
  memset(Auu, 0, 27 * nvx * sizeof(double));
  memset(Auv, 0, 27 * nvx * sizeof(double));
  memset(Avu, 0, 27 * nvx * sizeof(double));
  memset(Avv, 0, 27 * nvx * sizeof(double));
  memset(efvs, 0, (size_t)(nz - 1) * nx * ny * sizeof(double));
  if (dv) {  /* allocated and zeroed once per solve in the reference (:1155-1164) */
    memset(dv->omega_k, 0, (size_t)nz * nx * ny * sizeof(double));
    memset(dv->omega, 0, (size_t)nx * ny * sizeof(double));
  }
  double *eq = malloc((size_t)4 * (nz - 1) * sizeof(double));  /* efvs_qp(k,p) */
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!active_cell[IC(i, j)]) continue;
      double fl2 = 0.0;  /* vertical average, all cells (no mask) */
      for (int k = 1; k <= nz - 1; ++k)
        fl2 = fl2 + flwafact[IFL(k, i, j)] * (sigma[k] - sigma[k - 1]);
      double Kuu[4][4] = {{0}}, Kuv[4][4] = {{0}}, Kvu[4][4] = {{0}}, Kvv[4][4] = {{0}};
      double x[4], y[4], u[4], v[4], h[4], sx[4], sy[4], bx[4], by[4], efvs_qp[4];
      for (int n = 0; n < 4; ++n) {
        const int iv = i + ishift[2][n], jv = j + jshift[2][n];
        x[n] = xVertex[IV(iv, jv)];
        y[n] = yVertex[IV(iv, jv)];
        u[n] = u2[IV(iv, jv)];
        v[n] = v2[IV(iv, jv)];
        h[n] = stagthck[IV(iv, jv)];
        sx[n] = dusrf_dx ? dusrf_dx[IV(iv, jv)] : 0.0;
        sy[n] = dusrf_dy ? dusrf_dy[IV(iv, jv)] : 0.0;
        bx[n] = dv ? dv->btx[IV(iv, jv)] : 0.0;
        by[n] = dv ? dv->bty[IV(iv, jv)] : 0.0;
      }
      for (int p = 0; p < 4; ++p) {
        double ddx[4], ddy[4], detJ;
        if (basis_derivs_2d(x, y, p, ddx, ddy, &detJ) != ORC_OK) { free(eq); return ORC_ERR_SINGULAR_JAC; }
        if (approx == ORC_APPROX_L1L2) {
          double *ek = eq + (size_t)p * (nz - 1);
          effective_viscosity_l1l2(whichefvs, efvs_constant, nz, sigma, p, ddx, ddy, u, v, h, sx, sy,
                                   &flwa[IFL(1, i, j)], &flwafact[IFL(1, i, j)], rhoi, grav, ek);
          efvs_qp[p] = 0.0;
          for (int k = 1; k <= nz - 1; ++k) efvs_qp[p] = efvs_qp[p] + ek[k - 1] * (sigma[k] - sigma[k - 1]);
        } else if (approx == ORC_APPROX_DIVA) {
          double *ek = eq + (size_t)p * (nz - 1);
          double *e3 = dv->eq3 + (IC(i, j) * 4 + (size_t)p) * (size_t)(nz - 1);
          effective_viscosity_diva(whichefvs, efvs_constant, nz, sigma, p, ddx, ddy, u, v, bx, by,
                                   &flwafact[IFL(1, i, j)], e3);
          efvs_qp[p] = 0.0;
          for (int k = 1; k <= nz - 1; ++k) {
            ek[k - 1] = e3[k - 1];
            efvs_qp[p] = efvs_qp[p] + ek[k - 1] * (sigma[k] - sigma[k - 1]);
          }
        } else {
          efvs_qp[p] = effective_viscosity_ssa(whichefvs, efvs_constant, ddx, ddy, u, v, fl2);
          for (int k = 1; k <= nz - 1; ++k) eq[(size_t)p * (nz - 1) + k - 1] = efvs_qp[p];
        }
        double h_qp = 0.0;
        for (int n = 0; n < 4; ++n) h_qp = h_qp + phi2[n][p] * h[n];
        const double f = h_qp * efvs_qp[p] * wqp2[p] * detJ / vol0;
        for (int nc = 0; nc < 4; ++nc)
          for (int nr = 0; nr < 4; ++nr) {
            Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * ddx[nr] * ddx[nc] + ddy[nr] * ddy[nc]);
            Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * ddx[nr] * ddy[nc] + ddy[nr] * ddx[nc]);
            Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * ddy[nr] * ddx[nc] + ddx[nr] * ddy[nc]);
            Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * ddy[nr] * ddy[nc] + ddx[nr] * ddx[nc]);
          }
      }
      if (approx == ORC_APPROX_DIVA)
        integrals_diva(nz, sigma, dv->thck[IC(i, j)], eq, &dv->omega_k[IC(i, j) * (size_t)nz],
                       &dv->omega[IC(i, j)]);
      for (int k = 1; k <= nz - 1; ++k) {
        double e = 0.0;
        for (int p = 0; p < 4; ++p) e = e + eq[(size_t)p * (nz - 1) + k - 1];
        efvs[IFL(k, i, j)] = e / 4;
      }
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          if (fabs(Kuu[a][b] - Kuu[b][a]) > 1.0e-10) { free(eq); return ORC_ERR_ASYMMETRIC_ELEMENT; }
          if (fabs(Kvv[a][b] - Kvv[b][a]) > 1.0e-10) { free(eq); return ORC_ERR_ASYMMETRIC_ELEMENT; }
          if (fabs(Kuv[a][b] - Kvu[b][a]) > 1.0e-10) { free(eq); return ORC_ERR_ASYMMETRIC_ELEMENT; }
        }
      for (int nr = 0; nr < 4; ++nr) {
        const int ii = i + ishift[2][nr], jj = j + jshift[2][nr];
        for (int nc = 0; nc < 4; ++nc) {
          const size_t a = ((size_t)IV(ii, jj)) * 27 + (size_t)(indxA(ishift[nr][nc], jshift[nr][nc], 0) - 1);
          Auu[a] = Auu[a] + Kuu[nr][nc];
          Auv[a] = Auv[a] + Kuv[nr][nc];
          Avu[a] = Avu[a] + Kvu[nr][nc];
          Avv[a] = Avv[a] + Kvv[nr][nc];
        }
      }
    }
  free(eq);
  return ORC_OK;
}

/* compute_3d_velocity_L1L2 (:5834-6356), the vertex method (edge_velocity
 * = .false.): from the basal velocity (uvel, vvel)(nz,:,:) and the layer
 * viscosities of the last assembly, at cell centres the strain rates,
 * tau_parallel = 2 efvs eps_parallel and the integral of efvs from the top
 * of the column to the base of each layer; at the owned active vertices
 * the shear stresses tau_xz, tau_yz of each layer midpoint (the SIA stress
 * plus the horizontal gradients of the integrated membrane stresses,
 * glissade_gradient with the ice mask, margin 1) and the upward integral
 * u(k) = u(k+1) + 2 A tau_eff^2 (sigma(k+1) - sigma(k)) H tau_xz with A
 * and tau_parallel staggered over the ice cells (glissade_stagger margin
 * 1) and tau_eff^(n-1) = tau_eff^2 for n = 3.  Levels 1..nz-1 are zero
 * elsewhere; prescribed basal vertices keep the basal value on every
 * level.  Ends with the halo update (:3800-3801). */
static double grad_edges(double a, double b, int ma, int mb) {
  if (ma && mb) return (a + b) / 2.0;
  if (ma) return a;
  if (mb) return b;
  return 0.0;
}

/* glissade_gradient (glissade_grid_operators.F90:235-410) with
 * gradient_margin = 1: at each vertex the mean of the two edge differences
 * whose cells both hold ice, the one such edge, or zero. */
static void glissade_gradient_margin1(int nx, int ny, double dx, double dy, const double *f,
                                      double *df_dx, double *df_dy, const int *ice_mask) {
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const int sw = ice_mask[IC(i, j)], se = ice_mask[IC(i + 1, j)];
      const int nw = ice_mask[IC(i, j + 1)], ne = ice_mask[IC(i + 1, j + 1)];
      const double north = (f[IC(i + 1, j + 1)] - f[IC(i, j + 1)]) / dx;
      const double south = (f[IC(i + 1, j)] - f[IC(i, j)]) / dx;
      df_dx[IV(i, j)] = grad_edges(north, south, ne == 1 && nw == 1, se == 1 && sw == 1);
      const double east = (f[IC(i + 1, j + 1)] - f[IC(i + 1, j)]) / dy;
      const double west = (f[IC(i, j + 1)] - f[IC(i, j)]) / dy;
      df_dy[IV(i, j)] = grad_edges(east, west, ne == 1 && se == 1, nw == 1 && sw == 1);
    }
}

static void velocity_3d_l1l2(int nx, int ny, int nz, int nhalo, int periodic, const double *sigma,
                             double dx, double dy, const int *ice_mask, const int *active_cell,
                             const int *active_vertex, const int *umask_bed, const int *vmask_bed,
                             const double *xVertex, const double *yVertex, const double *thck,
                             const double *stagthck, const double *dusrf_dx,
                             const double *dusrf_dy, const double *flwa, const double *efvs,
                             double rhoi, double grav, double *uvel, double *vvel) {
  init_tables();
  const size_t nc = (size_t)nx * ny, nl = (size_t)(nz - 1), nvx = (size_t)(nx - 1) * (ny - 1);
  double *ux = calloc(nc, 8), *uy = calloc(nc, 8), *vx = calloc(nc, 8), *vy = calloc(nc, 8);
  double *tau_par = calloc(nl * nc, 8), *eint = calloc(nl * nc, 8);
  double *w1 = calloc(nc, 8), *w2 = calloc(nc, 8), *w3 = calloc(nc, 8), *lay = calloc(nc, 8);
  double *txz = calloc(nl * nvx, 8), *tyz = calloc(nl * nvx, 8);
  double *d1x = calloc(nvx, 8), *d1y = calloc(nvx, 8), *d2x = calloc(nvx, 8), *d2y = calloc(nvx, 8),
         *d3x = calloc(nvx, 8), *d3y = calloc(nvx, 8), *stp = calloc(nvx, 8), *stf = calloc(nvx, 8);
  const double dxr_ctr[4] = {-(1.0 - 0.0) / 4.0, (1.0 - 0.0) / 4.0, (1.0 + 0.0) / 4.0, -(1.0 + 0.0) / 4.0};
  const double dyr_ctr[4] = {-(1.0 - 0.0) / 4.0, -(1.0 + 0.0) / 4.0, (1.0 + 0.0) / 4.0, (1.0 - 0.0) / 4.0};
#define L3(k, i, j) (IC(i, j) * nl + ((size_t)(k) - 1))
#define LV(k, i, j) (IV(i, j) * nl + ((size_t)(k) - 1))
  for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
    for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
      if (!active_cell[IC(i, j)]) continue;
      double x[4], y[4], u[4], v[4], ddx[4], ddy[4], detJ;
      for (int n = 0; n < 4; ++n) {
        const int iv = i + ishift[2][n], jv = j + jshift[2][n];
        x[n] = xVertex[IV(iv, jv)];
        y[n] = yVertex[IV(iv, jv)];
        u[n] = uvel[IX(nz, iv, jv)];
        v[n] = vvel[IX(nz, iv, jv)];
      }
      basis_derivs_2d_at(x, y, dxr_ctr, dyr_ctr, ddx, ddy, &detJ);
      const size_t c = IC(i, j);
      for (int n = 0; n < 4; ++n) {
        ux[c] = ux[c] + ddx[n] * u[n];
        uy[c] = uy[c] + ddy[n] * u[n];
        vx[c] = vx[c] + ddx[n] * v[n];
        vy[c] = vy[c] + ddy[n] * v[n];
      }
      const double eps = sqrt(ux[c] * ux[c] + vy[c] * vy[c] + ux[c] * vy[c] +
                              0.25 * ((vx[c] + uy[c]) * (vx[c] + uy[c])));
      for (int k = 1; k <= nz - 1; ++k) tau_par[L3(k, i, j)] = 2.0 * efvs[IFL(k, i, j)] * eps;
      eint[L3(1, i, j)] = efvs[IFL(1, i, j)] * (sigma[1] - sigma[0]) * thck[c];
      for (int k = 2; k <= nz - 1; ++k)
        eint[L3(k, i, j)] = eint[L3(k - 1, i, j)] + efvs[IFL(k, i, j)] * (sigma[k] - sigma[k - 1]) * thck[c];
    }
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  for (int k = 1; k <= nz - 1; ++k) {
    for (size_t c = 0; c < nc; ++c) {
      w1[c] = eint[c * nl + k - 1] * (2.0 * ux[c] + vy[c]);
      w2[c] = eint[c * nl + k - 1] * (uy[c] + vx[c]);
      w3[c] = eint[c * nl + k - 1] * (2.0 * vy[c] + ux[c]);
    }
    glissade_gradient_margin1(nx, ny, dx, dy, w1, d1x, d1y, ice_mask);
    glissade_gradient_margin1(nx, ny, dx, dy, w2, d2x, d2y, ice_mask);
    glissade_gradient_margin1(nx, ny, dx, dy, w3, d3x, d3y, ice_mask);
    for (int j = jlo; j <= jhi; ++j)
      for (int i = ilo; i <= ihi; ++i) {
        const size_t w = IV(i, j);
        if (!active_vertex[w]) continue;
        const double depth = 0.5 * (sigma[k - 1] + sigma[k]) * stagthck[w];
        txz[LV(k, i, j)] = -rhoi * grav * depth * dusrf_dx[w] + 2.0 * d1x[w] + d2y[w];
        tyz[LV(k, i, j)] = -rhoi * grav * depth * dusrf_dy[w] + d2x[w] + 2.0 * d3y[w];
      }
  }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i)
      for (int k = 1; k <= nz - 1; ++k) { uvel[IX(k, i, j)] = 0.0; vvel[IX(k, i, j)] = 0.0; }
  for (int k = nz - 1; k >= 1; --k) {
    for (size_t c = 0; c < nc; ++c) lay[c] = tau_par[c * nl + k - 1];
    orc_stagger(nx, ny, lay, stp, ice_mask, 1);
    for (size_t c = 0; c < nc; ++c) lay[c] = flwa[c * nl + k - 1];
    orc_stagger(nx, ny, lay, stf, ice_mask, 1);
    for (int j = jlo; j <= jhi; ++j)
      for (int i = ilo; i <= ihi; ++i) {
        const size_t w = IV(i, j);
        if (!active_vertex[w]) continue;
        const double tx = txz[LV(k, i, j)], ty = tyz[LV(k, i, j)];
        const double tau_eff_sq = stp[w] * stp[w] + tx * tx + ty * ty;
        const double fact = 2.0 * stf[w] * tau_eff_sq * (sigma[k] - sigma[k - 1]) * stagthck[w];
        uvel[IX(k, i, j)] = umask_bed[w] == 1 ? uvel[IX(nz, i, j)] : uvel[IX(k + 1, i, j)] + fact * tx;
        vvel[IX(k, i, j)] = vmask_bed[w] == 1 ? vvel[IX(nz, i, j)] : vvel[IX(k + 1, i, j)] + fact * ty;
      }
  }
#undef L3
#undef LV
  orc_halo_stag(nx, ny, nz, periodic, uvel);
  orc_halo_stag(nx, ny, nz, periodic, vvel);
  free(ux); free(uy); free(vx); free(vy); free(tau_par); free(eint);
  free(w1); free(w2); free(w3); free(lay); free(txz); free(tyz);
  free(d1x); free(d1y); free(d2x); free(d2y); free(d3x); free(d3y); free(stp); free(stf);
}

/* compute_residual_velocity_2d (:9238-9351): no bed layer to leave out. */
static double residual_velocity_2d(int nx, int ny, int periodic, int whichresid,
                                   const double *u, const double *v,
                                   const double *usav, const double *vsav) {
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, periodic, &ilo, &ihi, &jlo, &jhi);
  double r = 0.0;
  long count = 0;
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i) {
      const size_t x = IV(i, j);
      const double speed = sqrt(u[x] * u[x] + v[x] * v[x]);
      if (speed != 0.0) {
        const double oldspeed = sqrt(usav[x] * usav[x] + vsav[x] * vsav[x]);
        const double diff = fabs((oldspeed - speed) / speed);
        if (whichresid == ORC_RESID_MEANU) { r = r + diff; ++count; }
        else if (diff > r) r = diff;
      }
    }
  if (whichresid == ORC_RESID_MEANU && count > 0) r = r / (double)count;
  return r;
}

/* One assembled 2-D system of the SSA or L1L2 branch at (u2, v2) (nx-1,ny-1): the
 * matrix in the kA = 0 slice of (27,1,nx-1,ny-1), b = the level-summed
 * load with the basal term and the Dirichlet rows of the bed level's
 * masks, halo-updated and symmetry-checked (:2703-2990). */
int orc_assemble_2d_system(const orc_model *m, const orc_setup *s, int approx,
                           const double *beta_internal, const double *u2,
                           const double *v2, double *efvs, double *Auu,
                           double *Auv, double *Avu, double *Avv, double *bu,
                           double *bv, long *nNonzeros) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1);
  if (approx != ORC_APPROX_SSA && approx != ORC_APPROX_L1L2) return ORC_ERR_ARGS;
  int st = assemble_2d(approx, nx, ny, nz, m->nhalo, s->sigma, s->active_cell, s->xVertex,
                       s->yVertex, u2, v2, s->stagthck, s->flwafact, m->flwa, s->dusrf_dx,
                       s->dusrf_dy, m->rhoi, m->grav, NULL, m->which_efvs, m->efvs_constant, efvs,
                       Auu, Auv, Avu, Avv);
  if (st != ORC_OK) return st;
  if (m->which_babc != ORC_BABC_NO_SLIP)
    basal_sliding_bc(nx, ny, 1, m->nhalo, m->dx, m->dy, s->active_cell, s->active_vertex,
                     beta_internal, s->xVertex, s->yVertex, m->which_assemble_beta, Auu, Avv);
  int *um = calloc(nvx, sizeof(int)), *vm = calloc(nvx, sizeof(int));
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const size_t w = IV(i, j);
      double lu = 0.0, lv = 0.0;
      for (int k = 1; k <= nz; ++k) {
        lu = lu + s->loadu[IX(k, i, j)];
        lv = lv + s->loadv[IX(k, i, j)];
      }
      bu[w] = lu;
      bv[w] = lv;
      um[w] = s->umask_dirichlet[IX(nz, i, j)];
      vm[w] = s->vmask_dirichlet[IX(nz, i, j)];
    }
  dirichlet_bc_3d(nx, ny, 1, m->nhalo, s->active_vertex, um, vm, u2, v2, Auu, Auv, Avu, Avv, bu, bv);
  free(um);
  free(vm);
  orc_halo_stag(nx, ny, 27, m->periodic, Auu);
  orc_halo_stag(nx, ny, 27, m->periodic, Auv);
  orc_halo_stag(nx, ny, 27, m->periodic, Avu);
  orc_halo_stag(nx, ny, 27, m->periodic, Avv);
  orc_halo_stag(nx, ny, 1, m->periodic, bu);
  orc_halo_stag(nx, ny, 1, m->periodic, bv);
  check_symmetry_assembled_3d(nx, ny, 1, m->periodic, s->active_vertex, Auu, Auv, Avu, Avv);
  *nNonzeros = count_nonzeros_3d(nx, ny, 1, m->periodic, s->active_vertex, Auu, Auv, Avu, Avv);
  return ORC_OK;
}

int orc_velocity_3d_l1l2(const orc_model *m, const orc_setup *s, const double *efvs,
                         double *uvel, double *vvel) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1);
  int *um = malloc(nvx * sizeof(int)), *vm = malloc(nvx * sizeof(int));
  for (size_t w = 0; w < nvx; ++w) {
    um[w] = s->umask_dirichlet[w * nz + (nz - 1)];
    vm[w] = s->vmask_dirichlet[w * nz + (nz - 1)];
  }
  velocity_3d_l1l2(nx, ny, nz, m->nhalo, m->periodic, s->sigma, m->dx, m->dy, s->ice_mask,
                   s->active_cell, s->active_vertex, um, vm, s->xVertex, s->yVertex, m->thck,
                   s->stagthck, s->dusrf_dx, s->dusrf_dy, m->flwa, efvs, m->rhoi, m->grav, uvel,
                   vvel);
  free(um);
  free(vm);
  return ORC_OK;
}

int orc_velo_2d_solve(const orc_model *m, int approx, double *uvel, double *vvel,
                      double *efvs, double *beta_internal, orc_stats *stats) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  if (approx != ORC_APPROX_SSA && approx != ORC_APPROX_L1L2) return ORC_ERR_ARGS;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1), n3 = nvx * nz, nA = nvx * 27;
  orc_setup s;
  orc_setup_alloc(m, &s);
  memset(stats, 0, sizeof(*stats));
  int st = orc_setup_solve(m, &s, uvel, vvel);
  if (st != ORC_OK) { orc_setup_free(&s); stats->status = st; return st; }
  double *Auu = xalloc(nA * 8), *Auv = xalloc(nA * 8), *Avu = xalloc(nA * 8),
         *Avv = xalloc(nA * 8), *bu = xalloc(nvx * 8), *bv = xalloc(nvx * 8),
         *u2 = xalloc(nvx * 8), *v2 = xalloc(nvx * 8), *us = xalloc(nvx * 8),
         *vs = xalloc(nvx * 8), *u3 = xalloc(n3 * 8), *v3 = xalloc(n3 * 8);
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      u2[IV(i, j)] = uvel[IX(nz, i, j)];  /* uvel_2d = uvel(nz,:,:) (:1179-1180) */
      v2[IV(i, j)] = vvel[IX(nz, i, j)];
    }
  int counter = 0;
  double outer_it_criterion = 1.0e10, outer_it_target = 1.0e-12;
  const double L2_target = 1.0e-4, L2_target_relative = 1.0e-7, resid_target = 1.0e-4;
  int status = ORC_OK;
  while (outer_it_criterion >= outer_it_target && counter < m->maxiter_nonlinear) {
    counter = counter + 1;
    for (size_t w = 0; w < nvx; ++w)  /* ubas = uvel_2d for SSA (:2236-2239) */
      for (int k = 1; k <= nz; ++k) { u3[w * nz + k - 1] = u2[w]; v3[w * nz + k - 1] = v2[w]; }
    st = orc_calcbeta(m, &s, u3, v3, beta_internal);
    if (st != ORC_OK) { status = st; break; }
    memcpy(us, u2, nvx * 8);
    memcpy(vs, v2, nvx * 8);
    long nnz = 0;
    st = orc_assemble_2d_system(m, &s, approx, beta_internal, u2, v2, efvs, Auu, Auv, Avu, Avv, bu,
                                bv, &nnz);
    if (st != ORC_OK) { status = st; break; }
    if (nnz == 0) {
      memset(u2, 0, nvx * 8);
      memset(v2, 0, nvx * 8);
      status = ORC_ZERO_MATRIX;
      break;
    }
    if (m->which_babc == ORC_BABC_NO_SLIP) {  /* frozen bed: u_2d = 0 (:3227-3240) */
      memset(u2, 0, nvx * 8);
      memset(v2, 0, nvx * 8);
      stats->L2_norm = 0.0;
      stats->L2_norm_relative = 0.0;
    } else {
      residual_vector_3d(nx, ny, 1, m->periodic, s.active_vertex, Auu, Auv, Avu, Avv, bu, bv, u2, v2,
                         &stats->L2_norm, &stats->L2_norm_relative);
      double err = 0.0;
      int niters = 0;
      if (m->which_sparse == ORC_SPARSE_PCG_CHRONGEAR)
        st = orc_pcg_chrongear_3d(nx, ny, 1, m->periodic, s.active_vertex, Auu, Auv, Avu, Avv, bu,
                                  bv, u2, v2, m->which_precond, m->pcg_maxiters, m->pcg_tol,
                                  m->pcg_ncheck, &err, &niters);
      else
        st = orc_pcg_standard_3d(nx, ny, 1, m->periodic, s.active_vertex, Auu, Auv, Avu, Avv, bu,
                                 bv, u2, v2, m->which_precond, m->pcg_maxiters, m->pcg_tol,
                                 m->pcg_ncheck, &err, &niters);
      stats->pcg_iters_total += niters;
      stats->pcg_iters_last = niters;
      stats->pcg_err_last = err;
      if (st == ORC_ERR_NAN) { status = st; break; }
    }
    orc_halo_stag(nx, ny, 1, m->periodic, u2);
    orc_halo_stag(nx, ny, 1, m->periodic, v2);
    const double resid_velo = residual_velocity_2d(nx, ny, m->periodic, m->which_resid, u2, v2, us, vs);
    stats->resid_velo = resid_velo;
    if (m->which_resid == ORC_RESID_L2NORM) {
      outer_it_criterion = stats->L2_norm; outer_it_target = L2_target;
    } else if (m->which_resid == ORC_RESID_L2NORM_RELATIVE) {
      outer_it_criterion = stats->L2_norm_relative; outer_it_target = L2_target_relative;
    } else {
      outer_it_criterion = resid_velo; outer_it_target = resid_target;
    }
  }
  /* SSA: uvel(k,:,:) = uvel_2d for every level (:3745-3750); L1L2:
   * uvel(nz,:,:) = uvel_2d and the 3-D reconstruction (:3759-3801) */
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i)
      for (int k = 1; k <= nz; ++k) {
        uvel[IX(k, i, j)] = u2[IV(i, j)];
        vvel[IX(k, i, j)] = v2[IV(i, j)];
      }
  if (approx == ORC_APPROX_L1L2 && (status == ORC_OK || status == ORC_ZERO_MATRIX))
    orc_velocity_3d_l1l2(m, &s, efvs, uvel, vvel);
  stats->picard_iters = counter;
  stats->converged = (status == ORC_OK && counter < m->maxiter_nonlinear) ? 1 : 0;
  if (status == ORC_OK && !stats->converged) status = ORC_WARN_PICARD_NOT_CONVERGED;
  stats->status = status;
  free(Auu); free(Auv); free(Avu); free(Avv); free(bu); free(bv);
  free(u2); free(v2); free(us); free(vs); free(u3); free(v3);
  orc_setup_free(&s);
  return status;
}

/* DIVA: the ice-plus-land mask of the setup (:1486-1496), with which
 * omega and omega_k are staggered. */
static void ice_plus_land(const orc_model *m, const orc_setup *s, int *ipl) {
  const size_t nc = (size_t)m->nx * m->ny;
  for (size_t c = 0; c < nc; ++c) ipl[c] = (s->ice_mask[c] == 1 || s->land_mask[c] == 1) ? 1 : 0;
}

/* One assembled DIVA system (:2703-2990) at the mean velocity (u2, v2):
 * the assembly updates efvs_qp_3d (eq3, in/out) from the basal traction
 * (btx, bty) and gives omega_k (nz,nx,ny) and omega (nx,ny); omega is
 * halo-updated and staggered over the ice-plus-land cells; beta_eff =
 * beta / (1 + beta stag_omega), or 1 / stag_omega on a no-slip bed (0
 * where stag_omega = 0) (Goldberg 2011 eq. 40-41, :2750-2790), enters the
 * basal term; then the bed level's Dirichlet rows, halo update and
 * symmetry check as for the other 2-D solves. */
int orc_assemble_diva_system(const orc_model *m, const orc_setup *s, const double *beta_internal,
                             const double *u2, const double *v2, const double *btx,
                             const double *bty, double *eq3, double *efvs, double *omega_k,
                             double *omega, double *beta_eff, double *Auu, double *Auv,
                             double *Avu, double *Avv, double *bu, double *bv, long *nNonzeros) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1), nc = (size_t)nx * ny;
  diva_state dv = {eq3, btx, bty, m->thck, omega_k, omega};
  int st = assemble_2d(ORC_APPROX_DIVA, nx, ny, nz, m->nhalo, s->sigma, s->active_cell, s->xVertex,
                       s->yVertex, u2, v2, s->stagthck, s->flwafact, m->flwa, NULL, NULL, m->rhoi,
                       m->grav, &dv, m->which_efvs, m->efvs_constant, efvs, Auu, Auv, Avu, Avv);
  if (st != ORC_OK) return st;
  orc_halo_cell_real(nx, ny, m->periodic, omega, 0.0, 0.0);
  int *ipl = malloc(nc * sizeof(int));
  double *so = malloc(nvx * sizeof(double));
  ice_plus_land(m, s, ipl);
  orc_stagger(nx, ny, omega, so, ipl, 1);
  for (size_t w = 0; w < nvx; ++w) {
    if (m->which_babc == ORC_BABC_NO_SLIP)
      beta_eff[w] = so[w] > 0.0 ? 1.0 / so[w] : 0.0;
    else
      beta_eff[w] = beta_internal[w] / (1.0 + beta_internal[w] * so[w]);
  }
  free(ipl);
  free(so);
  basal_sliding_bc(nx, ny, 1, m->nhalo, m->dx, m->dy, s->active_cell, s->active_vertex, beta_eff,
                   s->xVertex, s->yVertex, m->which_assemble_beta, Auu, Avv);
  int *um = calloc(nvx, sizeof(int)), *vm = calloc(nvx, sizeof(int));
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const size_t w = IV(i, j);
      double lu = 0.0, lv = 0.0;
      for (int k = 1; k <= nz; ++k) {
        lu = lu + s->loadu[IX(k, i, j)];
        lv = lv + s->loadv[IX(k, i, j)];
      }
      bu[w] = lu;
      bv[w] = lv;
      um[w] = s->umask_dirichlet[IX(nz, i, j)];
      vm[w] = s->vmask_dirichlet[IX(nz, i, j)];
    }
  dirichlet_bc_3d(nx, ny, 1, m->nhalo, s->active_vertex, um, vm, u2, v2, Auu, Auv, Avu, Avv, bu, bv);
  free(um);
  free(vm);
  orc_halo_stag(nx, ny, 27, m->periodic, Auu);
  orc_halo_stag(nx, ny, 27, m->periodic, Auv);
  orc_halo_stag(nx, ny, 27, m->periodic, Avu);
  orc_halo_stag(nx, ny, 27, m->periodic, Avv);
  orc_halo_stag(nx, ny, 1, m->periodic, bu);
  orc_halo_stag(nx, ny, 1, m->periodic, bv);
  check_symmetry_assembled_3d(nx, ny, 1, m->periodic, s->active_vertex, Auu, Auv, Avu, Avv);
  *nNonzeros = count_nonzeros_3d(nx, ny, 1, m->periodic, s->active_vertex, Auu, Auv, Avu, Avv);
  return ORC_OK;
}

/* The DIVA step after each linear solve (:3658-3696): the basal traction
 * beta_eff u_mean at every vertex, omega_k staggered over the
 * ice-plus-land cells level by level (no halo update first, as there),
 * and compute_3d_velocity_diva (:5730-5830) for the mean velocity
 * (diva_level_index = 0): at active vertices u(nz) = u_mean - tau_b
 * stag_omega, u(k) = u(nz) + tau_b stag_omega_k(k); then the halo update.
 * omega is taken halo-updated, as orc_assemble_diva_system leaves it. */
int orc_velocity_3d_diva(const orc_model *m, const orc_setup *s, const double *beta_eff,
                         const double *omega_k, const double *omega, const double *u2,
                         const double *v2, double *btx, double *bty, double *uvel,
                         double *vvel) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1), nc = (size_t)nx * ny;
  for (size_t w = 0; w < nvx; ++w) {
    btx[w] = beta_eff[w] * u2[w];
    bty[w] = beta_eff[w] * v2[w];
  }
  int *ipl = malloc(nc * sizeof(int));
  double *lay = malloc(nc * sizeof(double)), *sok = malloc(nvx * nz * sizeof(double)),
         *so = malloc(nvx * sizeof(double)), *t = malloc(nvx * sizeof(double));
  ice_plus_land(m, s, ipl);
  for (int k = 1; k <= nz; ++k) {
    for (size_t c = 0; c < nc; ++c) lay[c] = omega_k[c * nz + (k - 1)];
    orc_stagger(nx, ny, lay, t, ipl, 1);
    for (size_t w = 0; w < nvx; ++w) sok[w * nz + (k - 1)] = t[w];
  }
  orc_stagger(nx, ny, omega, so, ipl, 1);
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const size_t w = IV(i, j);
      if (!s->active_vertex[w]) continue;
      uvel[IX(nz, i, j)] = u2[w] - btx[w] * so[w];
      vvel[IX(nz, i, j)] = v2[w] - bty[w] * so[w];
      for (int k = 1; k <= nz - 1; ++k) {
        uvel[IX(k, i, j)] = uvel[IX(nz, i, j)] + btx[w] * sok[w * nz + (k - 1)];
        vvel[IX(k, i, j)] = vvel[IX(nz, i, j)] + bty[w] * sok[w * nz + (k - 1)];
      }
    }
  orc_halo_stag(nx, ny, nz, m->periodic, uvel);
  orc_halo_stag(nx, ny, nz, m->periodic, vvel);
  free(ipl); free(lay); free(sok); free(so); free(t);
  return ORC_OK;
}

/* glissade_velo_higher_solve, DIVA branch (whichapprox = HO_APPROX_DIVA):
 * the mean velocity (uvel_2d, vvel_2d: in, the last solve's; out, this
 * one's) from the 2-D system with beta_eff, the 3-D velocity and basal
 * traction (btractx, btracty: in/out) after every iteration, efvs (in:
 * the last solve's layer viscosities, the start of efvs_qp_3d, :1166-1170;
 * out: this solve's).  calcbeta reads the 3-D basal velocity (:2240-2243);
 * a no-slip bed enters through beta_eff, not the Dirichlet masks
 * (:1274-1278); Dirichlet columns start from the bed velocity (:1300-1303)
 * and inactive owned vertices from zero (:1700-1711). */
int orc_velo_diva_solve(const orc_model *m, double *uvel, double *vvel, double *uvel_2d,
                        double *vvel_2d, double *btractx, double *btracty, double *efvs,
                        double *beta_internal, orc_stats *stats) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const size_t nvx = (size_t)(nx - 1) * (ny - 1), nc = (size_t)nx * ny, nA = nvx * 27;
  orc_setup s;
  orc_setup_alloc(m, &s);
  memset(stats, 0, sizeof(*stats));
  int st = orc_setup_solve(m, &s, uvel, vvel);
  if (st != ORC_OK) { orc_setup_free(&s); stats->status = st; return st; }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      const size_t w = IV(i, j);
      const int kin = m->kinbcmask && m->kinbcmask[w] == 1;
      if (!kin) {  /* no bed mask for a no-slip DIVA solve */
        s.umask_dirichlet[IX(nz, i, j)] = 0;
        s.vmask_dirichlet[IX(nz, i, j)] = 0;
      } else {
        uvel_2d[w] = uvel[IX(nz, i, j)];
        vvel_2d[w] = vvel[IX(nz, i, j)];
      }
    }
  int ilo, ihi, jlo, jhi;
  owned_range(nx, ny, m->periodic, &ilo, &ihi, &jlo, &jhi);
  for (int j = jlo; j <= jhi; ++j)
    for (int i = ilo; i <= ihi; ++i)
      if (!s.active_vertex[IV(i, j)]) { uvel_2d[IV(i, j)] = 0.0; vvel_2d[IV(i, j)] = 0.0; }
  double *eq3 = xalloc((size_t)4 * (nz - 1) * nc * 8), *omk = xalloc((size_t)nz * nc * 8),
         *om = xalloc(nc * 8), *be = xalloc(nvx * 8);
  for (size_t c = 0; c < nc; ++c)
    for (int p = 0; p < 4; ++p)
      for (int k = 0; k < nz - 1; ++k) eq3[(c * 4 + p) * (nz - 1) + k] = efvs[c * (nz - 1) + k];
  double *Auu = xalloc(nA * 8), *Auv = xalloc(nA * 8), *Avu = xalloc(nA * 8),
         *Avv = xalloc(nA * 8), *bu = xalloc(nvx * 8), *bv = xalloc(nvx * 8),
         *us = xalloc(nvx * 8), *vs = xalloc(nvx * 8);
  int counter = 0;
  double outer_it_criterion = 1.0e10, outer_it_target = 1.0e-12;
  const double L2_target = 1.0e-4, L2_target_relative = 1.0e-7, resid_target = 1.0e-4;
  int status = ORC_OK;
  while (outer_it_criterion >= outer_it_target && counter < m->maxiter_nonlinear) {
    counter = counter + 1;
    st = orc_calcbeta(m, &s, uvel, vvel, beta_internal);  /* ubas = uvel(nz,:,:) */
    if (st != ORC_OK) { status = st; break; }
    memcpy(us, uvel_2d, nvx * 8);
    memcpy(vs, vvel_2d, nvx * 8);
    long nnz = 0;
    st = orc_assemble_diva_system(m, &s, beta_internal, uvel_2d, vvel_2d, btractx, btracty, eq3, efvs,
                                  omk, om, be, Auu, Auv, Avu, Avv, bu, bv, &nnz);
    if (st != ORC_OK) { status = st; break; }
    if (nnz == 0) {
      memset(uvel_2d, 0, nvx * 8);
      memset(vvel_2d, 0, nvx * 8);
      status = ORC_ZERO_MATRIX;
      break;
    }
    residual_vector_3d(nx, ny, 1, m->periodic, s.active_vertex, Auu, Auv, Avu, Avv, bu, bv, uvel_2d,
                       vvel_2d, &stats->L2_norm, &stats->L2_norm_relative);
    double err = 0.0;
    int niters = 0;
    if (m->which_sparse == ORC_SPARSE_PCG_CHRONGEAR)
      st = orc_pcg_chrongear_3d(nx, ny, 1, m->periodic, s.active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                                uvel_2d, vvel_2d, m->which_precond, m->pcg_maxiters, m->pcg_tol,
                                m->pcg_ncheck, &err, &niters);
    else
      st = orc_pcg_standard_3d(nx, ny, 1, m->periodic, s.active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                               uvel_2d, vvel_2d, m->which_precond, m->pcg_maxiters, m->pcg_tol,
                               m->pcg_ncheck, &err, &niters);
    stats->pcg_iters_total += niters;
    stats->pcg_iters_last = niters;
    stats->pcg_err_last = err;
    if (st == ORC_ERR_NAN) { status = st; break; }
    orc_halo_stag(nx, ny, 1, m->periodic, uvel_2d);
    orc_halo_stag(nx, ny, 1, m->periodic, vvel_2d);
    const double resid_velo =
        residual_velocity_2d(nx, ny, m->periodic, m->which_resid, uvel_2d, vvel_2d, us, vs);
    stats->resid_velo = resid_velo;
    orc_velocity_3d_diva(m, &s, be, omk, om, uvel_2d, vvel_2d, btractx, btracty, uvel, vvel);
    if (m->which_resid == ORC_RESID_L2NORM) {
      outer_it_criterion = stats->L2_norm; outer_it_target = L2_target;
    } else if (m->which_resid == ORC_RESID_L2NORM_RELATIVE) {
      outer_it_criterion = stats->L2_norm_relative; outer_it_target = L2_target_relative;
    } else {
      outer_it_criterion = resid_velo; outer_it_target = resid_target;
    }
  }
  stats->picard_iters = counter;
  stats->converged = (status == ORC_OK && counter < m->maxiter_nonlinear) ? 1 : 0;
  if (status == ORC_OK && !stats->converged) status = ORC_WARN_PICARD_NOT_CONVERGED;
  stats->status = status;
  free(eq3); free(omk); free(om); free(be);
  free(Auu); free(Auv); free(Avu); free(Avv); free(bu); free(bv); free(us); free(vs);
  orc_setup_free(&s);
  return status;
}

/* glissade_velo_higher_solve, 3-D Blatter-Pattyn branch with the native
 * PCG solvers (glissade_velo_higher.F90:654-3986). */
int orc_velo_higher_solve(const orc_model *m, double *uvel, double *vvel,
                          double *efvs, double *beta_internal,
                          orc_stats *stats) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  size_t n3 = (size_t)nz * (nx - 1) * (ny - 1), nA = n3 * 27;
  orc_setup s;
  orc_setup_alloc(m, &s);
  memset(stats, 0, sizeof(*stats));
  int st = orc_setup_solve(m, &s, uvel, vvel);
  if (st != ORC_OK) { orc_setup_free(&s); stats->status = st; return st; }
  double *Auu = xalloc(nA * 8), *Auv = xalloc(nA * 8), *Avu = xalloc(nA * 8),
         *Avv = xalloc(nA * 8), *bu = xalloc(n3 * 8), *bv = xalloc(n3 * 8),
         *usav = xalloc(n3 * 8), *vsav = xalloc(n3 * 8);
  int counter = 0;
  double outer_it_criterion = 1.0e10, outer_it_target = 1.0e-12;
  const double L2_target = 1.0e-4, L2_target_relative = 1.0e-7, resid_target = 1.0e-4;
  int status = ORC_OK;
  while (outer_it_criterion >= outer_it_target && counter < m->maxiter_nonlinear) {
    counter = counter + 1;
    st = orc_calcbeta(m, &s, uvel, vvel, beta_internal);
    if (st != ORC_OK) { status = st; break; }
    memcpy(usav, uvel, n3 * 8);
    memcpy(vsav, vvel, n3 * 8);
    long nnz = 0;
    st = orc_assemble_system(m, &s, beta_internal, uvel, vvel, efvs, Auu, Auv,
                             Avu, Avv, bu, bv, &nnz);
    if (st != ORC_OK) { status = st; break; }
    if (nnz == 0) {
      memset(uvel, 0, n3 * 8);
      memset(vvel, 0, n3 * 8);
      status = ORC_ZERO_MATRIX;
      break;
    }
    residual_vector_3d(nx, ny, nz, m->periodic, s.active_vertex, Auu, Auv, Avu,
                       Avv, bu, bv, uvel, vvel, &stats->L2_norm,
                       &stats->L2_norm_relative);
    double err = 0.0;
    int niters = 0;
    if (m->which_sparse == ORC_SPARSE_PCG_CHRONGEAR)
      st = orc_pcg_chrongear_3d(nx, ny, nz, m->periodic, s.active_vertex, Auu,
                                Auv, Avu, Avv, bu, bv, uvel, vvel,
                                m->which_precond, m->pcg_maxiters, m->pcg_tol,
                                m->pcg_ncheck, &err, &niters);
    else
      st = orc_pcg_standard_3d(nx, ny, nz, m->periodic, s.active_vertex, Auu,
                               Auv, Avu, Avv, bu, bv, uvel, vvel,
                               m->which_precond, m->pcg_maxiters, m->pcg_tol,
                               m->pcg_ncheck, &err, &niters);
    stats->pcg_iters_total += niters;
    stats->pcg_iters_last = niters;
    stats->pcg_err_last = err;
    if (st == ORC_ERR_NAN) { status = st; break; }
    orc_halo_stag(nx, ny, nz, m->periodic, uvel);
    orc_halo_stag(nx, ny, nz, m->periodic, vvel);
    double resid_velo = residual_velocity_3d(nx, ny, nz, m->periodic,
                                             m->which_resid, uvel, vvel, usav, vsav);
    stats->resid_velo = resid_velo;
    if (m->which_resid == ORC_RESID_L2NORM) {
      outer_it_criterion = stats->L2_norm; outer_it_target = L2_target;
    } else if (m->which_resid == ORC_RESID_L2NORM_RELATIVE) {
      outer_it_criterion = stats->L2_norm_relative; outer_it_target = L2_target_relative;
    } else {
      outer_it_criterion = resid_velo; outer_it_target = resid_target;
    }
  }
  stats->picard_iters = counter;
  stats->converged = (status == ORC_OK && counter < m->maxiter_nonlinear) ? 1 : 0;
  if (status == ORC_OK && !stats->converged) status = ORC_WARN_PICARD_NOT_CONVERGED;
  stats->status = status;
  free(Auu); free(Auv); free(Avu); free(Avv); free(bu); free(bv);
  free(usav); free(vsav);
  orc_setup_free(&s);
  return status;
}
