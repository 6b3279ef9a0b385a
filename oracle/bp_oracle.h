/*
 * bp_oracle.h -- CPU restatement of CISM's Blatter-Pattyn velocity solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the B200
 * solver: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product never links or calls it.
 *
 * Every routine follows the reference line by line on the reference's own
 * data layout: Fortran column-major arrays with a 2-cell halo (nhalo = 2),
 * cell fields (nx,ny), vertex fields (nx-1,ny-1), 3-D vectors
 * (nz,nx-1,ny-1) and the matrix blocks (27,nz,nx-1,ny-1).  Indices inside
 * the .c file are 1-based to match the Fortran.  Halo updates restate the
 * serial communication stub libglimmer/parallel_slap.F90 (periodic or
 * outflow global boundary).
 *
 * Parity pinning (the reference has no golden vectors and no Fortran
 * compiler exists here): reference invariants (sum phi = 1, sum dphi = 0,
 * element/assembled symmetry, detJ > 0), the analytic first-order slab
 * solution of tests/slab/plotSlab.py:143-157, and agreement between the
 * standard and Chronopoulos-Gear PCG on the same system.
 */
#ifndef BP_ORACLE_H
#define BP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Option values, libglide/glide_types.F90:198-263 */
enum {
  ORC_EFVS_CONSTANT = 0, ORC_EFVS_FLOWFACT = 1, ORC_EFVS_NONLINEAR = 2,
  ORC_BABC_BETA_CONSTANT = 0, ORC_BABC_BETA_EXTERNAL = 5, ORC_BABC_NO_SLIP = 6,
  ORC_RESID_MAXU = 0, ORC_RESID_MAXU_NO_UBAS = 1, ORC_RESID_MEANU = 2,
  ORC_RESID_L2NORM = 3, ORC_RESID_L2NORM_RELATIVE = 4,
  ORC_SPARSE_PCG_STANDARD = 2, ORC_SPARSE_PCG_CHRONGEAR = 3,
  ORC_PRECOND_NONE = 0, ORC_PRECOND_DIAG = 1, ORC_PRECOND_SIA = 2,
  ORC_GRADIENT_CENTERED = 0, ORC_GRADIENT_UPSTREAM1 = 1, ORC_GRADIENT_UPSTREAM2 = 2,
  ORC_GRADIENT_MARGIN_LAND = 0, ORC_GRADIENT_MARGIN_HYBRID = 1,
  ORC_GRADIENT_MARGIN_MARINE = 2,
  ORC_ASSEMBLE_STANDARD = 0, ORC_ASSEMBLE_LOCAL = 1,
  ORC_GROUND_NO_GLP = 0, ORC_GROUND_ALL = 2,
  ORC_APPROX_SSA = 1, ORC_APPROX_BP = 2, ORC_APPROX_L1L2 = 3, ORC_APPROX_DIVA = 4
};

/* Status codes shared with the product's C ABI. */
enum {
  ORC_OK = 0, ORC_ERR_NAN = 1, ORC_ERR_SINGULAR_JAC = 2,
  ORC_WARN_PCG_NOT_CONVERGED = 3, ORC_WARN_PICARD_NOT_CONVERGED = 4,
  ORC_ZERO_MATRIX = 5, ORC_ERR_ASYMMETRIC_ELEMENT = 8, ORC_ERR_BAD_BETA = 9,
  ORC_ERR_ARGS = 10
};

/* Velocity-dependent sliding laws of calcbeta (which_ho_babc values,
 * libglide/glide_types.F90:211-225) and the basal_physics fields they read
 * (libglide/glide_types.F90:1300-1370). */
enum {
  ORC_BABC_YIELD_PICARD = 2, ORC_BABC_PSEUDO_PLASTIC = 3, ORC_BABC_POWERLAW = 9,
  ORC_BABC_COULOMB_FRICTION = 10, ORC_BABC_COULOMB_POWERLAW_SCHOOF = 11,
  ORC_BABC_COULOMB_POWERLAW_TSAI = 12, ORC_BABC_POWERLAW_EFFECPRESS = 13
};
typedef struct {
  const double *effecpress_stag;      /* (nx-1,ny-1) Pa */
  const double *c_space_factor_stag;  /* (nx-1,ny-1) or NULL (= 1) */
  const double *mintauf_tau0;         /* (nx-1,ny-1) mintauf * tau0, Pa */
  double beta_powerlaw_umax;
  double powerlaw_c, powerlaw_m;
  double coulomb_c, coulomb_bump_max_slope, coulomb_bump_wavelength;
  double friction_powerlaw_k;
  double pseudo_plastic_q, pseudo_plastic_u0;
  double pseudo_plastic_phimin, pseudo_plastic_phimax;
  double pseudo_plastic_bedmin, pseudo_plastic_bedmax;
} orc_basal_physics;

/* Model state handed to the solve.  Sizes include the halo. */
typedef struct {
  int nx, ny, nz, nhalo;       /* nhalo must be 2 */
  int periodic;                /* 1 periodic global BC, 0 outflow */
  double dx, dy;
  const double *thck, *usrf, *topg;   /* (nx,ny), halo-filled, m */
  const double *flwa;                 /* (nz-1,nx,ny), Pa^-3 a^-1 */
  const double *beta_external;        /* (nx-1,ny-1), Pa a m^-1 */
  const int *kinbcmask;               /* (nx-1,ny-1) or NULL */
  double eus, thklim, max_slope, thck_gradient_ramp;
  double rhoi, rhoo, grav;
  double beta_const, beta_grounded_min, efvs_constant;
  int which_babc, which_efvs, which_resid, which_sparse, which_precond;
  int which_gradient, which_gradient_margin;
  int which_assemble_beta, which_assemble_taud, which_ground;
  int maxiter_nonlinear;
  int pcg_maxiters;            /* reference hard-codes 200 */
  double pcg_tol;              /* reference hard-codes 1e-8 */
  int pcg_ncheck;              /* reference hard-codes 5 */
  const orc_basal_physics *basal;  /* velocity-dependent laws, else NULL */
} orc_model;

typedef struct {
  int picard_iters;
  int pcg_iters_total;
  int pcg_iters_last;
  double pcg_err_last;
  double resid_velo;
  double L2_norm, L2_norm_relative;
  int converged;
  int status;
} orc_stats;

/* Glide sigma levels (libglide/glide_setup.F90:281-290, 375-382). */
void orc_sigma_glide(int nz, double *sigma, double *stagwbndsigma);

/* Halo updates restating libglimmer/parallel_slap.F90. */
void orc_halo_cell_real(int nx, int ny, int periodic, double *a,
                        double offset_ew, double offset_ns);
void orc_halo_stag(int nx, int ny, int nlead, int periodic, double *a);

/* Pre-step operators. */
void orc_get_masks(int nx, int ny, int periodic, const double *thck,
                   const double *topg, double eus, double thklim,
                   double rhoi, double rhoo, int *ice_mask,
                   int *floating_mask, int *ocean_mask, int *land_mask,
                   int *active_ice_mask);
void orc_stagger(int nx, int ny, const double *var, double *stagvar,
                 const int *mask, int stagger_margin);
void orc_surface_gradient(int nx, int ny, int periodic, double dx, double dy,
                          const int *active_ice_mask, const int *land_mask,
                          const double *usrf, const double *thck,
                          double thklim, double thck_gradient_ramp,
                          int ho_gradient, int ho_gradient_margin,
                          double max_slope, double *ds_dx, double *ds_dy);
void orc_grounded_fraction(int nx, int ny, const int *ice_mask,
                           const int *floating_mask, const int *land_mask,
                           int whichground, double *f_ground);

/* Pieces of the Picard iteration. */
int orc_assemble_3d(int nx, int ny, int nz, int nhalo, const double *sigma,
                    const int *active_cell, const double *xVertex,
                    const double *yVertex, const double *uvel,
                    const double *vvel, const double *stagusrf,
                    const double *stagthck, const double *flwafact,
                    int whichefvs, double efvs_constant, double *efvs,
                    double *Auu, double *Auv, double *Avu, double *Avv);
void orc_matvec_3d(int nx, int ny, int nz, int periodic,
                   const int *active_vertex, const double *Auu,
                   const double *Auv, const double *Avu, const double *Avv,
                   const double *xu, const double *xv, double *yu,
                   double *yv);
int orc_pcg_standard_3d(int nx, int ny, int nz, int periodic,
                        const int *active_vertex, const double *Auu,
                        const double *Auv, const double *Avu,
                        const double *Avv, const double *bu, const double *bv,
                        double *xu, double *xv, int precond, int maxiters,
                        double tolerance, int ncheck, double *err,
                        int *niters);
int orc_pcg_chrongear_3d(int nx, int ny, int nz, int periodic,
                         const int *active_vertex, const double *Auu,
                         const double *Auv, const double *Avu,
                         const double *Avv, const double *bu,
                         const double *bv, double *xu, double *xv,
                         int precond, int maxiters, double tolerance,
                         int ncheck, double *err, int *niters);

/* glissade_velo_higher_solve, 2-D branches (solve_2d, :1125-1128):
 * approx = ORC_APPROX_SSA, the depth-integrated velocity copied to every
 * level; ORC_APPROX_L1L2, the basal velocity of the L1L2 equations and the
 * 3-D velocity reconstructed from it. */
int orc_velo_2d_solve(const orc_model *m, int approx, double *uvel, double *vvel,
                      double *efvs, double *beta_internal, orc_stats *stats);

/* Post-solve diagnostics (glissade_velo_higher.F90:3847-3872). */
int orc_internal_stress(int nx, int ny, int nz, int nhalo, const double *sigma,
                        const int *active_cell, const double *xVertex,
                        const double *yVertex, const double *stagusrf,
                        const double *stagthck, const double *flwafact,
                        int whichefvs, double efvs_constant, const double *uvel,
                        const double *vvel, double *tau_xz, double *tau_yz,
                        double *tau_xx, double *tau_yy, double *tau_xy,
                        double *tau_eff);
int orc_internal_stress_approx(int nx, int ny, int nz, int nhalo, const double *sigma,
                               const int *active_cell, const double *xVertex,
                               const double *yVertex, const double *stagusrf,
                               const double *stagthck, const double *flwafact,
                               const double *efvs, int whichefvs, double efvs_constant,
                               int approx, const double *uvel, const double *vvel,
                               double *tau_xz, double *tau_yz, double *tau_xx, double *tau_yy,
                               double *tau_xy, double *tau_eff);
void orc_basal_friction_heatflx(int nx, int ny, int nz, int nhalo, int periodic,
                                const int *active_cell, const int *active_vertex,
                                const double *uvel, const double *vvel,
                                const double *beta, int which, double *bfricflx);

/* Boundary inputs computed by the setup part of glissade_velo_higher_solve
 * (libglissade/glissade_velo_higher.F90:987-2199).  Caller allocates. */
typedef struct {
  double *sigma, *stagwbndsigma;        /* nz, nz+1 */
  double *stagusrf, *stagthck;          /* (nx-1,ny-1) */
  double *dusrf_dx, *dusrf_dy;          /* (nx-1,ny-1) */
  double *xVertex, *yVertex;            /* (nx-1,ny-1) */
  double *f_ground;                     /* (nx-1,ny-1) */
  double *flwafact;                     /* (nz-1,nx,ny) */
  double *loadu, *loadv;                /* (nz,nx-1,ny-1) */
  int *active_cell;                     /* (nx,ny) */
  int *active_vertex;                   /* (nx-1,ny-1) */
  int *umask_dirichlet, *vmask_dirichlet; /* (nz,nx-1,ny-1) */
  int *ice_mask, *floating_mask, *ocean_mask, *land_mask; /* (nx,ny) */
} orc_setup;

void orc_setup_alloc(const orc_model *m, orc_setup *s);
void orc_setup_free(orc_setup *s);
int orc_setup_solve(const orc_model *m, orc_setup *s, double *uvel,
                    double *vvel);
/* beta_internal from calcbeta at basal velocity (uvel, vvel)(nz,:,:):
 * constant and external beta, and the velocity-dependent laws 2, 3, 9-13. */
int orc_calcbeta(const orc_model *m, const orc_setup *s, const double *uvel,
                 const double *vvel, double *beta_internal);
/* One assembled system of Picard iteration "counter": A, b after basal BC,
 * Dirichlet BC, halo update and the symmetry repair. */
int orc_assemble_system(const orc_model *m, const orc_setup *s,
                        const double *beta_internal, const double *uvel,
                        const double *vvel, double *efvs, double *Auu,
                        double *Auv, double *Avu, double *Avv, double *bu,
                        double *bv, long *nNonzeros);
/* One assembled 2-D system of the SSA or L1L2 branch (approx) at a 2-D
 * velocity ((nx-1,ny-1) arrays; the matrix in the kA = 0 slice of
 * (27,1,nx-1,ny-1)). */
int orc_assemble_2d_system(const orc_model *m, const orc_setup *s, int approx,
                           const double *beta_internal, const double *u2,
                           const double *v2, double *efvs, double *Auu,
                           double *Auv, double *Avu, double *Avv, double *bu,
                           double *bv, long *nNonzeros);
/* compute_3d_velocity_L1L2 and the halo update that follows it: levels
 * 1..nz-1 of (uvel, vvel) from the basal level nz and the layer
 * viscosities efvs (nz-1,nx,ny) of the last assembly. */
int orc_velocity_3d_l1l2(const orc_model *m, const orc_setup *s, const double *efvs,
                         double *uvel, double *vvel);
/* DIVA (Goldberg 2011): one assembled system at the mean velocity with
 * the traction (btx, bty); eq3 (nz-1,4,nx,ny) efvs_qp_3d in/out; outputs
 * efvs (nz-1,nx,ny), omega_k (nz,nx,ny), omega (nx,ny, halo-updated) and
 * beta_eff (nx-1,ny-1). */
int orc_assemble_diva_system(const orc_model *m, const orc_setup *s, const double *beta_internal,
                             const double *u2, const double *v2, const double *btx,
                             const double *bty, double *eq3, double *efvs, double *omega_k,
                             double *omega, double *beta_eff, double *Auu, double *Auv,
                             double *Avu, double *Avv, double *bu, double *bv, long *nNonzeros);
/* The step after a DIVA linear solve: traction, 3-D velocity, halo. */
int orc_velocity_3d_diva(const orc_model *m, const orc_setup *s, const double *beta_eff,
                         const double *omega_k, const double *omega, const double *u2,
                         const double *v2, double *btx, double *bty, double *uvel,
                         double *vvel);
/* Whole DIVA solve: uvel_2d, vvel_2d, btractx, btracty and efvs in/out. */
int orc_velo_diva_solve(const orc_model *m, double *uvel, double *vvel, double *uvel_2d,
                        double *vvel_2d, double *btractx, double *btracty, double *efvs,
                        double *beta_internal, orc_stats *stats);
/* Whole glissade_velo_higher_solve, 3-D Blatter-Pattyn branch. */
int orc_velo_higher_solve(const orc_model *m, double *uvel, double *vvel,
                          double *efvs, double *beta_internal,
                          orc_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
