// bp_kernels.h -- host-callable launchers of the device kernels.
#pragma once

#include <cuda_runtime.h>

#include "bp_common.h"

namespace bp {

enum MvMode { MV_INIT = 0, MV_STD_A = 1, MV_CG_FIRST = 2, MV_CG1 = 3, MV_CHECK = 4, MV_REFINE = 5 };

cudaError_t upload_ref_tables();

void launch_picard_begin(const DevView& v, cudaStream_t s);
void launch_save_usav(const DevView& v, cudaStream_t s);
// beta of the velocity-dependent sliding laws from the current velocity
// (and the corner betas of the standard basal assembly)
void launch_slide_beta(const DevView& v, cudaStream_t s);
void launch_assemble(const DevView& v, cudaStream_t s);
void launch_asm_qp(const DevView& v, cudaStream_t s);
void launch_asm_rows(const DevView& v, cudaStream_t s);
void launch_rhs(const DevView& v, cudaStream_t s);
// L1L2: the 3-D velocity v.x3 from the basal velocity v.x and the layer
// viscosities v.efvs of the last assembly
void launch_l1l2_velocity(const DevView& v, cudaStream_t s);
// DIVA: omega and beta_eff after assembly pass 1; the traction and 3-D
// velocity v.x3 after the linear solve
void launch_diva_beta(const DevView& v, cudaStream_t s);
void launch_diva_velocity(const DevView& v, cudaStream_t s);
// Residual modes (MV_INIT, MV_CHECK, MV_REFINE) run with (minb, grid_cap),
// the Krylov matvecs (MV_STD_A, MV_CG_FIRST, MV_CG1) with (minb_k, grid_k).
void launch_mv(int mode, const DevView& v, cudaStream_t s);
// CTAs of the Krylov matvec of this mode, storage and occupancy target
// (0, 4, 6) that fit on one SM at once (0 on error).
int krylov_resident_ctas(const DevView& v, int mode, int minb);
void launch_std_update(bool check, const DevView& v, cudaStream_t s);
void launch_std_dir(const DevView& v, cudaStream_t s);
void launch_cg_first_update(const DevView& v, cudaStream_t s);
void launch_cg_update(bool check, const DevView& v, cudaStream_t s);
void launch_picard_check(const DevView& v, cudaStream_t s);
// Condition of a device-resident WHILE loop (graph conditional handle h):
// *iter counts the passes (reset: set to 0); h = 1 while the counter
// v.cnt->picard_active (picard) or pcg_active is positive and *iter < cap.
void launch_loop_cond(cudaGraphConditionalHandle h, const DevView& v, bool picard, int* iter, int cap, bool reset,
                      cudaStream_t s);
// Programmatic dependent launch of the PCG kernels on (default) or off,
// for the launches of the calling thread.
void set_pdl(bool on);
void launch_make_a32(const DevView& v, cudaStream_t s);
// The SIA column preconditioner's factors (v.sia_f) of the solving
// instances that use it, from the assembled matrix.
void launch_sia_factor(const DevView& v, cudaStream_t s);
void launch_matvec_plain(const DevView& v, const double2* x, double2* y, cudaStream_t s);
void launch_dinv(const DevView& v, int precond, cudaStream_t s);
void launch_bb(const DevView& v, cudaStream_t s);
// element stresses into tau[6][nelem] and the basal frictional heat flux
// into bf ([ncells] for which_bfric 0, [ncols] for 1); either may be null
void launch_diagnostics(const DevView& v, int which_bfric, double* tau, double* bf, cudaStream_t s);
// a shallow-shelf solve's 2-D solution on each of L levels, x3 [ncols][L]
void launch_levels_from_2d(const DevView& v, double2* x3, int L, cudaStream_t s);
// cell_beta from col_beta (0 at a corner without a column), every cell
void launch_corner_beta(const DevView& v, cudaStream_t s);
// store: 0 full FP64, 1 symmetric FP64, 2 symmetric FP32; minb: 0, 6 or 8
// resident CTAs per SM; grid: CTAs (0 = one per tile).  -1 if unavailable.
int launch_tune_mv(int store, int minb, int grid, const DevView& v, cudaStream_t s);

}  // namespace bp
