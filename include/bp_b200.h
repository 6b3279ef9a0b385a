/*
 * bp_b200.h -- C ABI of the B200 Blatter-Pattyn velocity solver.
 *
 * Drop-in replacement for the body of CISM's Picard loop in
 * glissade_velo_higher_solve (libglissade/glissade_velo_higher.F90:2206-3727)
 * and for its native PCG solvers (libglissade/glissade_velo_higher_pcg.F90),
 * selected on the Fortran side by a new which_ho_sparse value (5).
 *
 * Conventions
 *  - Every array is in the reference's Fortran column-major layout on the
 *    local grid with a 2-cell halo (nhalo = 2): cell fields (nx,ny), vertex
 *    fields (nx-1,ny-1), 3-D velocity fields (nz,nx-1,ny-1), matrix blocks
 *    (27,nz,nx-1,ny-1) with the stencil index fastest (indxA_3d: iA fastest,
 *    then jA, then kA; diagonal = 14 in 1-based numbering).
 *  - Units are the solver's internal ones: m, m/a, Pa a, Pa^-3 a^-1; the
 *    matrix is scaled by vol0 = 1e9 m^3 as in the reference.
 *  - Integer masks are 0/1 ints.  Host arrays are owned by the caller and
 *    only read/written during the call.
 *  - All entry points return a bp_status code (0 = success).  Codes 3 and 4
 *    are warnings: the output is valid but not converged, as the reference
 *    continues after the same conditions (glissade_velo_higher_pcg.F90:542-547,
 *    glissade_velo_higher.F90:3731-3745).
 *  - Calls on one context are serialised by the caller (no re-entrancy);
 *    distinct contexts may be used from distinct threads.
 */
#ifndef BP_B200_H
#define BP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define BP_ABI_VERSION 6

typedef struct bp_ctx bp_ctx;

typedef enum {
  BP_OK = 0,
  BP_ERR_NAN = 1,              /* alpha/eta NaN, glissade_velo_higher_pcg.F90:397-399, 460-463 */
  BP_ERR_SINGULAR_JAC = 2,     /* glissade_velo_higher.F90:6458-6473 */
  BP_WARN_PCG_NOT_CONVERGED = 3,
  BP_WARN_PICARD_NOT_CONVERGED = 4,
  BP_ZERO_MATRIX = 5,          /* all-zero matrix: velocity zeroed, :3191-3220 */
  BP_ERR_CUDA = 6,
  BP_ERR_BUDGET = 7,           /* device iteration budget exhausted */
  BP_ERR_BAD_BETA = 9,         /* glissade_basal_traction.F90:567-579 */
  BP_ERR_ARGS = 10,
  BP_ERR_NO_DEVICE = 11
} bp_status;

typedef enum { BP_FP64 = 0, BP_MIXED = 1 } bp_precision;

/* Start of the Picard loop: the caller's velocity (as the reference, which
 * starts from the last time step's, glissade.F90:1919-1987), or the
 * learned guess of the network loaded by bp_guess_load. */
typedef enum { BP_GUESS_GIVEN = 0, BP_GUESS_LEARNED = 1 } bp_guess_mode;

/* Velocity-dependent sliding law: calcbeta
 * (libglissade/glissade_basal_traction.F90:67-598) evaluated on the device
 * at the start of every Picard iteration from the basal velocity
 * (uvel, vvel)(nz,:,:), where the reference calls it
 * (glissade_velo_higher.F90:2502-2517).  law is the which_ho_babc value
 * (libglide/glide_types.F90:211-225):
 *    2 yield stress (Picard)   beta = tau_y / |u|                  (:266-277)
 *    3 pseudo-plastic          beta = tan(phi) N / (u0^q s^(1-q))  (:207-264)
 *    9 power law               beta = C s^(1/m - 1)                (:357-363)
 *   10 Coulomb friction (Schoof 2005)                               (:384-424)
 *   11 Coulomb / power law (Schoof, MISMIP+)                        (:426-470)
 *   12 Coulomb / power law (Tsai et al. 2015)                       (:472-509)
 *   13 power law with effective pressure (p = 3, q = 1)            (:365-382)
 * s = sqrt(u^2 + v^2 + 0.01^2) m/a (:181), capped at beta_powerlaw_umax
 * when that is > 0 (:187-189); law 2 uses the uncapped sqrt(u^2 + v^2 + 0.01^2).  phi of law 3
 * varies linearly with topg - eus between bedmin and bedmax; law 10 uses
 * the basal-layer flow factor staggered over ice cells.  beta is then
 * multiplied by f_ground, raised to beta_grounded_min where f_ground > 0
 * (:538-566), and must be >= 0 (else BP_ERR_BAD_BETA, :570-582).  Vertex
 * fields are (nx-1,ny-1); a field the law does not read may be NULL. */
typedef struct {
  int law;
  const double *f_ground;            /* grounded fraction, :55-178 of glissade_grounding_line.F90 */
  const double *effecpress_stag;     /* N, Pa (laws 3, 10-13) */
  const double *c_space_factor_stag; /* law 10 (NULL: 1) */
  const double *flwa_basal_stag;     /* Pa^-3 a^-1 (law 10) */
  const double *yield_stress;        /* tau_y = mintauf * tau0, Pa (law 2) */
  const double *topg;                /* (nx,ny) m, read at the vertex's (i,j) as the reference does (law 3) */
  double eus;                        /* m (law 3) */
  double beta_grounded_min;          /* Pa a/m */
  double beta_powerlaw_umax;         /* m/a, 0 = no cap */
  double powerlaw_c, powerlaw_m;
  double coulomb_c, coulomb_bump_max_slope, coulomb_bump_wavelength;
  double friction_powerlaw_k;        /* law 13 */
  double pseudo_plastic_q, pseudo_plastic_u0;
  double pseudo_plastic_phimin, pseudo_plastic_phimax;   /* degrees */
  double pseudo_plastic_bedmin, pseudo_plastic_bedmax;   /* m */
} bp_sliding;

/* Fields of the L1L2 solve (whichapprox = HO_APPROX_L1L2) beyond the
 * shallow-shelf ones.  The layer viscosities of
 * compute_effective_viscosity_L1L2 (glissade_velo_higher.F90:7382-7618)
 * read the flow factor, the surface gradient and the thickness; the 3-D
 * velocity reconstruction compute_3d_velocity_L1L2 (:5834-6356) the cell
 * thickness and the same gradient.  The reconstruction's ice mask is taken
 * as active_cell, which it equals at every owned vertex under the default
 * which_ho_calving_front (active_ice_mask = ice_mask). */
typedef struct {
  const double *thck;                 /* (nx,ny) m */
  const double *flwa;                 /* (nz-1,nx,ny) Pa^-3 a^-1 */
  const double *dusrf_dx, *dusrf_dy;  /* (nx-1,ny-1) surface gradient of the setup (:1582) */
  double rhoi, grav;                  /* kg m^-3, m s^-2 */
} bp_l1l2;

/* State of the DIVA solve (whichapprox = HO_APPROX_DIVA, after Goldberg
 * 2011; glissade_velo_higher.F90:2742-2857, 3658-3696, 5601-5830,
 * 7622-7864).  The 2-D system is solved for the depth-mean velocity with
 * the basal term beta_eff = beta / (1 + beta omega) (1 / omega on a
 * no-slip bed); the layer viscosities come from the last iteration's
 * vertical shear, tau_b sigma / efvs_old; after every linear solve the
 * basal traction tau_b = beta_eff u_mean and the 3-D velocity u(k) =
 * u_mean - tau_b omega + tau_b omega_k(k) are formed, and the next
 * iteration's sliding law reads that 3-D basal velocity.  The mean
 * velocity, the traction and the viscosities carry over from one solve to
 * the next, so the arrays below are read on entry and (uvel_2d, vvel_2d,
 * btractx, btracty) written back with the result.  The setup leaves a
 * Dirichlet column's mean velocity at its basal velocity (:1300-1303) and
 * zeroes it at owned inactive vertices (:1700-1711); a no-slip bed sets no
 * basal Dirichlet mask here (:1274-1278). */
typedef struct {
  double *uvel_2d, *vvel_2d;         /* (nx-1,ny-1) m/a, mean velocity: in the last solve's, out this one's */
  double *btractx, *btracty;         /* (nx-1,ny-1) Pa, basal traction: in/out */
  const double *efvs;                /* (nz-1,nx,ny) Pa a, the last solve's layer viscosities (0 = none),
                                        halo-updated as the reference's caller leaves them (a periodic
                                        halo cell's omega is computed from its own values; the
                                        reference copies its image's, equal for such inputs) */
  const double *thck;                /* (nx,ny) m */
  const int *ice_plus_land_mask;     /* (nx,ny), the staggering mask of omega (:1486-1496) */
} bp_diva;

/* Boundary inputs of one solve: what the setup part of
 * glissade_velo_higher_solve (:987-2199) has computed when the Picard loop
 * starts (:2206).  beta_internal is the calcbeta result for the
 * velocity-independent laws (constant or external beta); with a
 * velocity-dependent law (sliding != NULL) beta is recomputed on the device
 * every Picard iteration and beta_internal is not read. */
typedef struct {
  int nx, ny, nz, nhalo;        /* local grid incl. halo; nhalo must be 2 */
  int periodic;                 /* 1: periodic global BC (serial default), 0: outflow */
  double dx, dy;                /* m */
  const double *sigma;          /* nz */
  const double *stagusrf;       /* (nx-1,ny-1) m */
  const double *stagthck;       /* (nx-1,ny-1) m */
  const double *beta_internal;  /* (nx-1,ny-1) Pa a/m */
  const double *flwafact;       /* (nz-1,nx,ny) 0.5*A^(-1/n), :1919-1939 */
  const int *active_cell;       /* (nx,ny), get_vertex_geometry :4163-4313 */
  const int *active_vertex;     /* (nx-1,ny-1) */
  const double *loadu, *loadv;  /* (nz,nx-1,ny-1) load vector, :2024-2111 */
  const int *umask_dirichlet;   /* (nz,nx-1,ny-1), :1270-1324 */
  const int *vmask_dirichlet;   /* (nz,nx-1,ny-1) */
  /* options (values of libglide/glide_types.F90:198-263) */
  int which_babc;               /* 6 = no-slip (no basal term); else basal term from beta */
  int which_efvs;               /* 0 constant, 1 flow factor, 2 nonlinear */
  double efvs_constant;         /* Pa a */
  int which_assemble_beta;      /* 0 standard (2x2 face quadrature), 1 local */
  int which_resid;              /* 0..4, :3716-3725 */
  int pcg_variant;              /* 2 standard PCG, 3 Chronopoulos-Gear */
  int which_precond;            /* 0 none, 1 diagonal, 2 SIA column */
  int maxiter_nonlinear;        /* Picard cap, default 100 */
  int pcg_maxiters;             /* reference: 200 */
  int pcg_ncheck;               /* reference: 5 */
  double pcg_tol;               /* reference: 1e-8 */
  int precision;                /* bp_precision */
  double inner_tol;             /* BP_MIXED: residual reduction of one refinement cycle
                                   (FP32-matrix Krylov solve between two FP64
                                   residuals; <= 0: 1e-4) */
  const bp_sliding *sliding;    /* NULL: beta_internal, fixed over the Picard loop */
  int approx_2d;                /* the 2-D solves (solve_2d, :1125-1128), one unknown
                                   pair per column: 1 shallow-shelf (HO_APPROX_SSA),
                                   the result copied to every level; 3 L1L2
                                   (HO_APPROX_L1L2), the basal velocity and the 3-D
                                   velocity reconstructed from it (needs l1l2);
                                   4 DIVA (HO_APPROX_DIVA), the mean velocity and
                                   the 3-D velocity (needs diva).  0: the 3-D
                                   Blatter-Pattyn solve.  Shared by a batch; the
                                   2-D solves take which_precond 0 or 1 */
  const bp_l1l2 *l1l2;          /* approx_2d = 3 only */
  const bp_diva *diva;          /* approx_2d = 4 only; its outputs are written by
                                   bp_solve, bp_batch_solve and bp_problem_get */
  int guess_mode;               /* bp_guess_mode; BP_GUESS_LEARNED (the 3-D solve
                                   only) replaces uvel/vvel on entry by the network's
                                   guess, computed on the device; needs bp_guess_load */
} bp_inputs;

typedef struct {
  int status;
  int picard_iters;
  int pcg_iters_total;          /* inner iterations for BP_MIXED */
  int pcg_iters_last;
  int refine_steps_total;       /* BP_MIXED outer refinement steps */
  int converged;                /* Picard converged */
  double pcg_err_last;          /* |b-Ax|/|b| of the last linear solve */
  double resid_velo;            /* last Picard velocity criterion */
  double L2_norm, L2_norm_relative; /* |Ax-b| before the last linear solve */
  float ms_upload, ms_assemble, ms_pcg, ms_total;
  double h2d_bytes, d2h_bytes;  /* host<->device bytes moved by this call */
} bp_stats;

/* Context: one CUDA device, one stream, persistent device buffers. */
int bp_create(int device, bp_ctx **ctx);
int bp_destroy(bp_ctx *ctx);
const char *bp_last_error(const bp_ctx *ctx);
int bp_abi_version(void);

/* Whole Picard loop of glissade_velo_higher_solve on the device
 * (replaces :2206-3727 when which_ho_sparse = 5).  uvel/vvel are the
 * initial guess on input and the solution on output (nz,nx-1,ny-1); efvs
 * (nz-1,nx,ny) receives the element-averaged viscosity (:5167-5172).  Any
 * of efvs/stats may be NULL. */
int bp_solve(bp_ctx *ctx, const bp_inputs *in, double *uvel, double *vvel,
             double *efvs, bp_stats *stats);

/* n independent solves in one set of launches (uneven grid sizes allowed,
 * common nz, pcg_variant and pcg_ncheck).  Arrays of n pointers. */
int bp_batch_solve(bp_ctx *ctx, int n, const bp_inputs *in,
                   double *const *uvel, double *const *vvel,
                   double *const *efvs, bp_stats *stats);

/* Linear solve only, on an assembled system (drop-in for the calls of
 * pcg_solver_standard_3d / pcg_solver_chrongear_3d at
 * glissade_velo_higher.F90:3329-3356).  variant 2 = standard, 3 =
 * Chronopoulos-Gear; precond 0/1/2.  xu/xv: initial guess in, solution out. */
int bp_pcg(bp_ctx *ctx, int nx, int ny, int nz, int periodic,
           const int *active_vertex, const double *Auu, const double *Auv,
           const double *Avu, const double *Avv, const double *bu,
           const double *bv, double *xu, double *xv, int precond, int variant,
           double tol, int maxiters, int ncheck, int precision,
           double *err, int *niters);

/* y = A x on owned active rows (matvec_multiply_structured_3d,
 * glissade_velo_higher_pcg.F90:2533-2647); other rows of y are zero. */
int bp_matvec(bp_ctx *ctx, int nx, int ny, int nz, int periodic,
              const int *active_vertex, const double *Auu, const double *Auv,
              const double *Avu, const double *Avv, const double *xu,
              const double *xv, double *yu, double *yv);

/* One assembled system at velocity (uvel, vvel): assembly, basal BC and
 * Dirichlet BC (:3003-3119).  Rows of owned active vertices are filled;
 * all other rows are zero.  Any output may be NULL. */
int bp_assemble(bp_ctx *ctx, const bp_inputs *in, const double *uvel,
                const double *vvel, double *Auu, double *Auv, double *Avu,
                double *Avv, double *bu, double *bv, double *efvs);

/* Residual resid = A x - b on owned active rows, with |A x - b|, |b| and
 * their ratio in norms[0..2] -- without allocating any device memory.
 * No counterpart in the reference: it is for callers that own all device
 * memory themselves (a fixed pool, or code that must not hit the implicit
 * device synchronisation of cudaMalloc/cudaFree inside a time step).
 * Every pointer is a DEVICE pointer in the reference layout above (halo
 * included, x halo-consistent); stream is a cudaStream_t (NULL = default).
 * Work is enqueued on the stream and not waited for.  The reduction scratch
 * is a fixed file-scope device array shared by all calls: at most
 * nz*(nx-1)*(ny-1) = 16,777,216 rows (larger: BP_ERR_ARGS); calls that
 * overlap on the GPU race on it and must be serialised; the first call on
 * a device, and the first after its context was made again (e.g. after
 * cudaDeviceReset), looks up the array's address and should precede any
 * stream capture. */
int bp_residual_noalloc(int nx, int ny, int nz, int periodic,
                        const int *active_vertex, const double *Auu,
                        const double *Auv, const double *Avu, const double *Avv,
                        const double *xu, const double *xv, const double *bu,
                        const double *bv, double *resid_u, double *resid_v,
                        double *norms, void *stream);

/* ------------------------------------------------------------------
 * Resident problems: the compiled inputs of one solve (or a batch) kept
 * in device memory across runs, e.g. for repeated solves on one geometry.
 * The reference has no counterpart (it recomputes everything per call);
 * bp_solve is bp_problem_create + set_guess + run + get + destroy.
 * ------------------------------------------------------------------ */
typedef struct bp_problem bp_problem;

/* ------------------------------------------------------------------
 * Learned initial guess.  No counterpart in the reference, whose Picard
 * loop starts from the velocity the caller passes (glissade.F90:1919-1987
 * keeps the last time step's).  bp_guess_load reads the weights of a
 * trained U-Net (the .bin file beside cism_b200/weights/unet_marine.npz)
 * into the context; then an input with guess_mode = BP_GUESS_LEARNED
 * starts from the network's estimate of the velocity, computed on the
 * device from that input's own device data (thickness, gravity load, beta,
 * active vertices) and written straight into the solve's initial guess.
 * The solve itself is unchanged and converges to the same tolerances.
 * Returns BP_ERR_ARGS (message in bp_last_error) for a missing or
 * malformed file.
 * ------------------------------------------------------------------ */
int bp_guess_load(bp_ctx *ctx, const char *path);
/* Kernels launched by the network since the context was created. */
int bp_guess_launches(bp_ctx *ctx);

int bp_problem_create(bp_ctx *ctx, int n, const bp_inputs *in, bp_problem **out);
/* Upload an initial guess (n arrays (nz,nx-1,ny-1)); it is kept on the
 * device and restored at the start of every bp_problem_run.  Instances
 * whose inputs set guess_mode = BP_GUESS_LEARNED take the network's guess
 * instead, formed on the device (their array pointers may be NULL). */
int bp_problem_set_guess(bp_problem *p, double *const *uvel, double *const *vvel);
/* The stored initial guess of each instance, scattered like the solution
 * (3-D solves). */
int bp_problem_get_guess(bp_problem *p, double *const *uvel, double *const *vvel);
/* Run the Picard solve from the stored guess entirely on device data;
 * stats (array of n, may be NULL) are filled at the end. */
int bp_problem_run(bp_problem *p, bp_stats *stats);
/* Copy the solution (and efvs if non-NULL) back to the host. */
int bp_problem_get(bp_problem *p, double *const *uvel, double *const *vvel,
                   double *const *efvs);
int bp_problem_destroy(bp_problem *p);
/* Post-solve diagnostics of glissade_velo_higher_solve (:3847-3872),
 * computed on the device at the solution of the last bp_problem_run, per
 * instance (arrays of n pointers; any may be NULL):
 *  - compute_internal_stress (:6968-7195): the stresses tau_xz, tau_yz,
 *    tau_xx, tau_yy, tau_xy and tau_eff (Pa) at element centres,
 *    (nz-1,nx,ny), zero outside active cells, from the 3-D velocity; the
 *    branch of the solve's approximation (:7100-7147: shallow-shelf
 *    horizontal gradients and viscosity, L1L2 the layer viscosity, else
 *    the 3-D ones);
 *  - compute_basal_friction_heatflx (:6755-6964): bfricflx (W/m^2) at cell
 *    centres (nx,ny), by the finite-element face quadrature
 *    (which_bfric = 0) or at vertices unstaggered to cells (1, the
 *    reference's default which_ho_assemble_bfric), with the beta_internal
 *    of the last Picard iteration and the 3-D basal velocity. */
int bp_problem_diagnostics(bp_problem *p, int which_bfric, double *const *tau_xz,
                           double *const *tau_yz, double *const *tau_xx,
                           double *const *tau_yy, double *const *tau_xy,
                           double *const *tau_eff, double *const *bfricflx);

/* Kernel timing with CUDA events on the solver's stream, per category, for
 * the runs made while enabled (CUDA graphs are bypassed while enabled).
 * Categories: 0 FP64 PCG matvec, 1 FP64 PCG vector update, 2 FP64
 * residual check, 3 FP32 inner matvec, 4 FP32 inner update, 5 assembly
 * pass 1, 6 assembly pass 2, 7 right-hand side, 8 other. */
#define BP_NUM_KERNEL_CATEGORIES 9
int bp_problem_timing(bp_problem *p, int enable);
/* Device-side wall clock of a region of work on the context's stream:
 * CUDA events recorded at start and stop (ms). */
int bp_timer_start(bp_ctx *ctx);
int bp_timer_stop(bp_ctx *ctx, float *ms);
int bp_problem_kernel_times(bp_problem *p, double *ms, int *launches);
/* Time reps launches of a plain y = A x kernel on the problem's current
 * matrix (run the problem once first): store 0 full FP64 rows, 1 symmetric
 * FP64, 2 symmetric FP32; minb = resident CTAs per SM the kernel is
 * compiled for (0, 6, 8); grid = CTAs (0 = one per tile).  ms = mean per
 * launch.  BP_ERR_ARGS if the variant does not match the storage. */
int bp_problem_tune_mv(bp_problem *p, int store, int minb, int grid, int reps, float *ms);
/* Nodes that went through FP64 and FP32 Krylov matvecs during the last
 * timing run, and the autotuner's choice for those matvecs (occupancy
 * target in resident CTAs per SM, grid; 0 = none / one CTA per tile). */
int bp_problem_mv_nodes(bp_problem *p, double *fp64_nodes, double *fp32_nodes,
                        int *minb, int *grid);
/* Node count and, per FP64 matvec launch, the algorithmic bytes moved. */
int bp_problem_info(bp_problem *p, long *nodes, long *active_columns,
                    long *elements, double *matvec_bytes_fp64,
                    double *matvec_bytes_fp32);

/* ------------------------------------------------------------------
 * Host-side mirror of the setup part of glissade_velo_higher_solve, for
 * callers that hold the model fields rather than the boundary inputs.
 * ------------------------------------------------------------------ */
typedef struct {
  int nx, ny, nz, nhalo, periodic;
  double dx, dy;
  const double *thck, *usrf, *topg;   /* (nx,ny) halo-filled, m */
  const double *flwa;                 /* (nz-1,nx,ny) Pa^-3 a^-1 */
  const double *beta_external;        /* (nx-1,ny-1) Pa a/m */
  const int *kinbcmask;               /* (nx-1,ny-1) or NULL */
  double eus, thklim, max_slope, thck_gradient_ramp;
  double rhoi, rhoo, grav;
  double beta_const, beta_grounded_min, efvs_constant;
  int which_babc, which_efvs, which_resid, which_sparse, which_precond;
  int which_gradient, which_gradient_margin;
  int which_assemble_beta, which_assemble_taud, which_ground;
  int maxiter_nonlinear, pcg_maxiters, pcg_ncheck;
  double pcg_tol;
  int precision;
  double inner_tol;
  /* velocity-dependent sliding law (which_babc = sliding->law), or NULL;
   * bp_setup computes its f_ground and flwa_basal_stag and takes topg, eus
   * and beta_grounded_min from this struct's fields above */
  const bp_sliding *sliding;
  int approx_2d;                /* as in bp_inputs; bp_setup fills the L1L2 fields */
  /* DIVA: the carried-over state (uvel_2d, vvel_2d, btractx, btracty,
   * efvs; thck and the mask are filled by bp_setup, which also applies the
   * Dirichlet and inactive-vertex rules to uvel_2d, vvel_2d) */
  const bp_diva *diva;
} bp_model;

/* Caller-allocated outputs of the setup (sizes as in bp_inputs). */
typedef struct {
  double *sigma;                   /* nz */
  double *stagusrf, *stagthck;     /* (nx-1,ny-1) */
  double *beta_internal;           /* (nx-1,ny-1) */
  double *flwafact;                /* (nz-1,nx,ny) */
  int *active_cell;                /* (nx,ny) */
  int *active_vertex;              /* (nx-1,ny-1) */
  double *loadu, *loadv;           /* (nz,nx-1,ny-1) */
  int *umask_dirichlet, *vmask_dirichlet; /* (nz,nx-1,ny-1) */
  /* with a sliding law only: outputs f_ground and, for law 10,
   * flwa_basal_stag ((nx-1,ny-1) each), and the law handed to the solve */
  double *f_ground, *flwa_basal_stag;
  bp_sliding sliding;
  /* L1L2 only: outputs the surface gradient ((nx-1,ny-1) each) and the
   * L1L2 fields handed to the solve */
  double *dusrf_dx, *dusrf_dy;
  bp_l1l2 l1l2;
  /* DIVA only: outputs the ice-plus-land mask ((nx,ny)) and the DIVA
   * state handed to the solve */
  int *ice_plus_land_mask;
  bp_diva diva;
} bp_setup_arrays;

/* Masks, staggering, surface gradient, vertex geometry, flow factor, load
 * vector and calcbeta (:1270-2199, :2502-2517); zeroes uvel/vvel at owned
 * inactive vertices (:1700-1711).  Fills *in to point at the arrays. */
int bp_setup(const bp_model *m, bp_setup_arrays *out, double *uvel,
             double *vvel, bp_inputs *in);

/* bp_setup followed by bp_solve. */
int bp_velo_higher_solve(bp_ctx *ctx, const bp_model *m, double *uvel,
                         double *vvel, double *efvs, bp_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
