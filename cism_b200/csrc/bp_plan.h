// bp_plan.h -- host-side compilation of reference-layout inputs into the
// compact column/element form used by the device kernels (pure C++, no CUDA).
#pragma once

#include <string>
#include <vector>

#include "bp_b200.h"
#include "bp_common.h"

namespace bp {

// Locally owned vertex range of the serial build (parallel_slap.F90:655-673),
// 1-based Fortran indices into the (nx-1, ny-1) vertex grid.
struct OwnedRange {
  int ilo, ihi, jlo, jhi;
};
OwnedRange owned_range(int nx, int ny, int periodic);

// Owned image of a halo'd vertex index (1-based) or -1 when the vertex lies
// outside the global domain (outflow).  Periodic: the staggered halo update
// copies vertex V-2 -> 1, V-1 -> 2 and 3 -> V (V = n-1 vertices).
int vertex_image(int i, int n, int periodic);

struct HostPlan {
  int nz = 0, ninst = 0;   // nz: levels of the solve (1 for the 2-D solves)
  int nz_out = 0;          // levels of the velocity arrays (the model's nz)
  bool solve2d = false;    // 2-D solve: shallow-shelf or L1L2
  bool l1l2 = false;       // L1L2 (the 3-D velocity reconstructed after the loop)
  bool diva = false;       // DIVA (3-D velocity, traction and point viscosities every iteration)
  int nefvs = 0;           // length of the element viscosity array (L1L2: ncells * (nz_out - 1))
  int ncols = 0, nnodes = 0, npad = 0, ncells = 0, nelem = 0, ntiles = 0;
  int W = 1, lsh = 0;      // column block width and log2 (bp_common.h: node layout)
  std::vector<InstParams> inst;
  std::vector<int> col_inst, col_nbr, col_cells, col_ij;
  std::vector<int> col_node, col_nbn;  // node of (col, 0); the neighbours' col_node [9][ncols]
  std::vector<double> col_beta;
  std::vector<double> col_slide;  // [3][ncols] (f_ground, c1, c2) when any instance has a sliding law
  bool any_sliding = false;
  std::vector<double2> load;
  std::vector<uint8_t> dmask;
  std::vector<int> cell_inst, cell_ij, cell_cols;
  std::vector<double> cell_s, cell_h, cell_beta, flwafact;
  std::vector<double> cell_flwa, cell_thck, cell_ds, col_ds;  // L1L2 only (cell_thck: DIVA too)
  std::vector<double> col_h;  // stagthck at the column's vertex (L1L2, the learned guess)
  std::vector<double> flwafact_layers;  // shallow-shelf: [ncells][nz_out-1], for the element stresses
  // DIVA only: starting point viscosities [ncells][4][nl], mean velocity
  // and traction [ncols], the columns' ice-plus-land bits, and each
  // instance's state arrays (written back with the result)
  std::vector<double> eq3_0;
  std::vector<double2> x2d_0, col_bt0;
  std::vector<uint8_t> col_ipl;
  std::vector<bp_diva> diva_io;
  std::vector<int> tile_start, tile_end, tile_inst, tile_ncols, tile_col0;
  std::vector<int> guess_mode;  // per instance, bp_guess_mode
  // per-instance grid sizes, for scatters
  std::vector<int> nx, ny, periodic;
};

// Node of (col, k) (the blocked level-major layout of bp_common.h).
inline size_t node_of(const HostPlan& p, int col, int k) {
  return (size_t)p.col_node[col] + ((size_t)k << p.lsh);
}

// Columns only (matrix-level entry points): fills columns, neighbours and
// tiles of one instance; cells are left empty.
bool build_column_plan(int nx, int ny, int nz, int periodic,
                       const int* active_vertex, HostPlan* plan,
                       std::string* err);

// Checks a velocity-dependent sliding law and forms its per-instance
// constants (SlideParams); false with *err when the law or a field it
// needs is missing.
bool slide_params(const bp_sliding& L, SlideParams* sp, std::string* err);
// The two per-vertex products of the law at vertex (i,j) (1-based) of an
// instance with nx cells in x (SlideParams).
void slide_vertex(const bp_sliding& L, int i, int j, int nx, double* c1, double* c2);

// Full plan for n solves.
bool build_plan(const bp_inputs* in, int n, HostPlan* plan, std::string* err);

// velocity (nz,nx-1,ny-1) of instance b <-> node vector
void gather_velocity(const HostPlan& p, int b, const double* uvel,
                     const double* vvel, double2* x);
void scatter_velocity(const HostPlan& p, int b, const double2* x,
                      double* uvel, double* vvel);
// DIVA: the 3-D velocity [ncols][nz_out] of instance b from the bed level
// of (uvel, vvel) (the first iteration's sliding law reads it)
void gather_velocity_3d(const HostPlan& p, int b, const double* uvel,
                        const double* vvel, double2* x3);
// DIVA: the mean velocity x and traction bt [ncols] of instance b into its
// bp_diva arrays (zero away from the columns, then the halo update)
void scatter_diva(const HostPlan& p, int b, const double2* x, const double2* bt);
// L1L2: the reconstructed velocity [ncols][nz_out] of instance b -> uvel,
// vvel (nz,nx-1,ny-1), zero on levels 1..nz-1 away from the columns, then
// the halo update (glissade_velo_higher.F90:3773-3801)
void scatter_velocity_3d(const HostPlan& p, int b, const double2* x3,
                         double* uvel, double* vvel);
// element-averaged viscosity -> efvs (nz-1,nx,ny), zero elsewhere
void scatter_efvs(const HostPlan& p, int b, const double* efvs_elem,
                  double* efvs);
// matrix blocks (27,nz,nx-1,ny-1) -> device layout [2][27][npad] of (u,v) pairs
void gather_matrix(const HostPlan& p, const double* Auu, const double* Auv,
                   const double* Avu, const double* Avv, double2* A);
void scatter_matrix(const HostPlan& p, const double2* A, double* Auu,
                    double* Auv, double* Avu, double* Avv);
// symmetric storage [2][14][npad] -> full rows (lower half from neighbours)
void scatter_matrix_sym(const HostPlan& p, const double2* A, double* Auu,
                        double* Auv, double* Avu, double* Avv);
// full rows -> symmetric storage (upper offsets only)
void gather_matrix_sym(const HostPlan& p, const double* Auu, const double* Auv,
                       const double* Avu, const double* Avv, double2* A);
void scatter_vector(const HostPlan& p, int b, const double2* v, double* vu,
                    double* vv);

// staggered_parallel_halo for an (nlead, nx-1, ny-1) field.
void halo_stag(int nx, int ny, int nlead, int periodic, double* a);
// parallel_halo for an (nx, ny) cell field (parallel_slap.F90:1790-1860).
void halo_cells(int nx, int ny, int periodic, double* a);

// Elements of the post-solve diagnostics: cells x (nz_out - 1) layers (the
// 3-D elements of any solve, 2-D ones included).
inline int diagnostic_elements(const HostPlan& p) { return p.ncells * (p.nz_out - 1); }
// The device view of the post-solve diagnostics of a 2-D solve: the 3-D
// elements over the nz_out levels, the 3-D velocity x3 [ncols][nz_out]
// and, for the shallow-shelf solve, the per-layer flow factor
// (flwafact_layers on the device); x3's node of (col, k) is col * nz_out + k,
// so col_node3 holds col * nz_out per column.  A 3-D solve's view is
// returned as is.
DevView diagnostics_view(const DevView& v, const HostPlan& p, double2* x3, const double* flwafact_layers,
                         const int* col_node3);

// Post-solve diagnostics of instance b to the reference layout: nv element
// fields vals[v][nelem] -> out[v] (nz-1,nx,ny), zero outside active cells
// (a null out[v] is skipped); the basal frictional heat flux (nx,ny) from
// active-cell values (which = 0) or column values unstaggered to the cells
// with glissade_unstagger margin 0 (which = 1,
// glissade_grid_operators.F90:152-231), then the cell halo update
// (glissade_velo_higher.F90:6960).
void scatter_elements(const HostPlan& p, int b, const double* vals, int nv,
                      double* const* out);
void scatter_bfric(const HostPlan& p, int b, int which, const double* vals,
                   double* bfricflx);

}  // namespace bp
