// bp_plan.cpp -- compile reference-layout inputs into the compact device form.
#include "bp_plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace bp {

namespace {

inline size_t vtx(int i, int j, int nx) { return (size_t)(j - 1) * (nx - 1) + (i - 1); }
inline size_t cel(int i, int j, int nx) { return (size_t)(j - 1) * nx + (i - 1); }

int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Column ids of the owned active vertices of one instance.
struct ColumnMap {
  int nx, ny, periodic;
  std::vector<int> id;  // (nx-1)*(ny-1), -1 where not an owned active vertex
  int lookup(int i, int j) const {
    int ii = vertex_image(i, nx, periodic), jj = vertex_image(j, ny, periodic);
    if (ii < 0 || jj < 0) return -1;
    return id[vtx(ii, jj, nx)];
  }
};

void add_columns(int nx, int ny, int nz, int periodic, const int* active_vertex,
                 int inst_index, HostPlan* p, ColumnMap* cm,
                 std::vector<std::pair<int, int>>* cols_ij) {
  OwnedRange R = owned_range(nx, ny, periodic);
  cm->nx = nx; cm->ny = ny; cm->periodic = periodic;
  cm->id.assign((size_t)(nx - 1) * (ny - 1), -1);
  for (int j = R.jlo; j <= R.jhi; ++j)
    for (int i = R.ilo; i <= R.ihi; ++i)
      if (active_vertex[vtx(i, j, nx)]) {
        cm->id[vtx(i, j, nx)] = p->ncols + (int)cols_ij->size();
        cols_ij->push_back({i, j});
      }
  (void)nz;
  (void)inst_index;
}

// Blocks of W consecutive columns of instance b, one tile each (W * nz <=
// kTile nodes, whole columns, so a CTA can run the column solves of the SIA
// preconditioner on its own tile); sets the columns' nodes and the
// instance's tile and node ranges.
void add_tiles(HostPlan* p, int b, int col_begin, int ncols) {
  const int W = p->W, span = W * p->nz;
  InstParams& ip = p->inst[b];
  ip.tile_begin = (int)p->tile_start.size();
  ip.node_begin = ip.tile_begin * span;
  for (int c0 = 0; c0 < ncols; c0 += W) {
    const int t = (int)p->tile_start.size();
    p->tile_start.push_back(t * span);
    p->tile_end.push_back((t + 1) * span);
    p->tile_inst.push_back(b);
    p->tile_ncols.push_back(std::min(W, ncols - c0));
    p->tile_col0.push_back(col_begin + c0);
    for (int c = c0; c < std::min(ncols, c0 + W); ++c) p->col_node[col_begin + c] = t * span + (c - c0);
  }
  ip.tile_end = (int)p->tile_start.size();
  ip.node_end = ip.tile_end * span;
}

// The neighbours' nodes at level 0, after every column has its node.
void fill_nbn(HostPlan* p) {
  const size_t NC = (size_t)p->ncols;
  p->col_nbn.resize(9 * NC);
  for (size_t i = 0; i < 9 * NC; ++i) p->col_nbn[i] = p->col_nbr[i] >= 0 ? p->col_node[p->col_nbr[i]] : -1;
}

void set_block_width(HostPlan* p) {
  p->W = block_width(p->nz);
  p->lsh = 0;
  while ((1 << p->lsh) < p->W) ++p->lsh;
}

}  // namespace

OwnedRange owned_range(int nx, int ny, int periodic) {
  OwnedRange r;
  r.ilo = periodic ? 3 : 2;
  r.jlo = periodic ? 3 : 2;
  r.ihi = nx - 2;
  r.jhi = ny - 2;
  return r;
}

int vertex_image(int i, int n, int periodic) {
  const int V = n - 1;
  if (periodic) {
    const int P = n - 4;  // owned vertices per row
    if (i < 1 || i > V) return -1;
    int t = ((i - 3) % P + P) % P;
    return t + 3;
  }
  return (i >= 2 && i <= n - 2) ? i : -1;
}

bool build_column_plan(int nx, int ny, int nz, int periodic,
                       const int* active_vertex, HostPlan* p,
                       std::string* err) {
  if (nx < 6 || ny < 6 || nz < 2 || nz > kNzMax) {
    *err = "grid too small or nz out of range";
    return false;
  }
  *p = HostPlan();
  p->nz = nz;
  p->nz_out = nz;
  set_block_width(p);
  p->ninst = 1;
  p->inst.resize(1);
  std::memset(&p->inst[0], 0, sizeof(InstParams));
  p->nx = {nx}; p->ny = {ny}; p->periodic = {periodic};
  ColumnMap cm;
  std::vector<std::pair<int, int>> cols;
  add_columns(nx, ny, nz, periodic, active_vertex, 0, p, &cm, &cols);
  const int nc = (int)cols.size();
  p->ncols = nc;
  p->nnodes = nc * nz;
  p->col_node.assign(nc, 0);
  p->col_inst.assign(nc, 0);
  p->col_ij.resize(2 * (size_t)nc);
  p->col_nbr.resize(9 * (size_t)nc);
  p->col_cells.assign(4 * (size_t)nc, -1);
  p->col_beta.assign(nc, 0.0);
  for (int c = 0; c < nc; ++c) {
    int i = cols[c].first, j = cols[c].second;
    p->col_ij[c] = i;
    p->col_ij[nc + c] = j;
    for (int jA = -1; jA <= 1; ++jA)
      for (int iA = -1; iA <= 1; ++iA)
        p->col_nbr[(size_t)((jA + 1) * 3 + (iA + 1)) * nc + c] = cm.lookup(i + iA, j + jA);
  }
  InstParams& ip = p->inst[0];
  ip.col_begin = 0; ip.col_end = nc;
  add_tiles(p, 0, 0, nc);
  fill_nbn(p);
  p->ntiles = (int)p->tile_start.size();
  p->npad = round_up(std::max(p->ntiles * p->W * nz, 1), 64);
  p->load.assign(p->npad, double2{0.0, 0.0});
  p->dmask.assign(p->npad, 0);
  return true;
}

// calcbeta's velocity-dependent laws (glissade_basal_traction.F90:67-598):
// the factors that do not depend on the speed, in the reference's order of
// evaluation.  gn = 3 is an integer in the reference (glimmer_physcon.F90:75),
// so N**gn is a product and 1/gn a real division; the law with effective
// pressure fixes p = 3, q = 1 (:378-379); pi is glimmer_physcon's literal.
bool slide_params(const bp_sliding& L, SlideParams* sp, std::string* err) {
  std::memset(sp, 0, sizeof(*sp));
  const bool needN = L.law == 3 || (L.law >= 10 && L.law <= 13);
  if (L.law != 2 && L.law != 3 && !(L.law >= 9 && L.law <= 13)) {
    *err = "sliding law must be 2, 3 or 9-13 (velocity-dependent which_ho_babc)";
    return false;
  }
  if (!L.f_ground || (needN && !L.effecpress_stag) || (L.law == 2 && !L.yield_stress) ||
      (L.law == 3 && !L.topg) || (L.law == 10 && !L.flwa_basal_stag)) {
    *err = "sliding law: missing input field";
    return false;
  }
  if ((L.law >= 9 && L.law <= 12 && L.law != 10 && !(L.powerlaw_m > 0.0)) ||
      (L.law == 10 && !(L.coulomb_bump_max_slope > 0.0))) {
    *err = "sliding law: powerlaw_m and coulomb_bump_max_slope must be > 0";
    return false;
  }
  sp->law = L.law;
  sp->umax = L.beta_powerlaw_umax;
  sp->bmin = L.beta_grounded_min;
  const double m = L.powerlaw_m;
  switch (L.law) {
    case 3:
      sp->k = std::pow(L.pseudo_plastic_u0, L.pseudo_plastic_q);
      sp->e1 = 1.0 - L.pseudo_plastic_q;
      break;
    case 9:
      sp->c = L.powerlaw_c;
      sp->e2 = 1.0 / m - 1.0;
      break;
    case 10:
      sp->e1 = 1.0 / 3 - 1.0;
      sp->e2 = -1.0 / 3;
      break;
    case 11:
      sp->k = std::pow(L.powerlaw_c, m);
      sp->e1 = 1.0 / m;
      sp->e2 = 1.0 / m - 1.0;
      break;
    case 12:
      sp->c = L.powerlaw_c;
      sp->e1 = 1.0 / m;
      break;
    case 13:
      sp->e1 = 1.0 / 3.0 - 1.0;
      break;
    default:
      break;
  }
  return true;
}

void slide_vertex(const bp_sliding& L, int i, int j, int nx, double* c1, double* c2) {
  const size_t v = vtx(i, j, nx);
  const double N = L.effecpress_stag ? L.effecpress_stag[v] : 0.0;
  *c1 = 0.0;
  *c2 = 0.0;
  switch (L.law) {
    case 2:
      *c1 = L.yield_stress[v];
      break;
    case 3: {  // :225-247, phi from topg(ew,ns) read at the vertex's indices
      const double pi = 3.14159265358979;
      const double bed = L.topg[cel(i, j, nx)] - L.eus;
      double phi;
      if (bed <= L.pseudo_plastic_bedmin) phi = L.pseudo_plastic_phimin;
      else if (bed >= L.pseudo_plastic_bedmax) phi = L.pseudo_plastic_phimax;
      else
        phi = L.pseudo_plastic_phimin + ((bed - L.pseudo_plastic_bedmin) /
                                         (L.pseudo_plastic_bedmax - L.pseudo_plastic_bedmin)) *
                                            (L.pseudo_plastic_phimax - L.pseudo_plastic_phimin);
      const double tanphi = std::tan(phi * pi / 180.0);
      *c1 = tanphi * N;
      break;
    }
    case 10: {  // :400-418
      const double cs = L.c_space_factor_stag ? L.c_space_factor_stag[v] : 1.0;
      const double big_lambda = (L.coulomb_bump_wavelength / L.coulomb_bump_max_slope) * L.flwa_basal_stag[v];
      *c1 = L.coulomb_c * cs * N;
      *c2 = N * N * N * big_lambda;
      break;
    }
    case 11:  // :446-451
      *c1 = L.powerlaw_c * L.coulomb_c * N;
      *c2 = std::pow(L.coulomb_c * N, L.powerlaw_m);
      break;
    case 12:  // :490
      *c1 = L.coulomb_c * N;
      break;
    case 13:  // :380-382
      *c1 = std::pow(L.friction_powerlaw_k, -1.0 / 3.0) * std::pow(N, 1.0 / 3.0);
      break;
    default:
      break;
  }
}

bool build_plan(const bp_inputs* in, int n, HostPlan* p, std::string* err) {
  if (n < 1 || !in) { *err = "no instances"; return false; }
  *p = HostPlan();
  const int nz_in = in[0].nz;
  if (nz_in < 2 || nz_in > kNzMax) { *err = "nz out of range (2..64)"; return false; }
  // the 2-D solves (shallow-shelf, L1L2) have one unknown pair per column
  // (solve_2d, glissade_velo_higher.F90:1125-1128)
  const int approx = in[0].approx_2d;
  if (approx != 0 && approx != 1 && approx != 3 && approx != 4) {
    *err = "approx_2d must be 0, 1 (SSA), 3 (L1L2) or 4 (DIVA)";
    return false;
  }
  const bool solve2d = approx != 0, l1l2 = approx == 3, diva = approx == 4;
  const int nz = solve2d ? 1 : nz_in, nl = nz_in - 1;
  p->nz = nz;
  p->nz_out = nz_in;
  set_block_width(p);
  p->solve2d = solve2d;
  p->l1l2 = l1l2;
  p->diva = diva;
  p->ninst = n;
  p->inst.resize(n);
  std::vector<std::vector<std::pair<int, int>>> cols(n);
  std::vector<ColumnMap> cms(n);
  std::vector<std::vector<std::pair<int, int>>> cells(n);
  // pass 1: columns and cells of every instance
  for (int b = 0; b < n; ++b) {
    const bp_inputs& I = in[b];
    if (I.nz != nz_in) { *err = "all instances of a batch must share nz"; return false; }
    if (I.approx_2d != approx) { *err = "all instances of a batch must share the approximation"; return false; }
    if (solve2d && I.which_precond == 2) {
      *err = "the 2-D solves take which_precond 0 or 1";
      return false;
    }
    if (l1l2 && (!I.l1l2 || !I.l1l2->thck || !I.l1l2->flwa || !I.l1l2->dusrf_dx || !I.l1l2->dusrf_dy)) {
      *err = "the L1L2 solve needs l1l2 with thck, flwa, dusrf_dx and dusrf_dy";
      return false;
    }
    if (diva && (!I.diva || !I.diva->uvel_2d || !I.diva->vvel_2d || !I.diva->btractx || !I.diva->btracty ||
                 !I.diva->thck || !I.diva->ice_plus_land_mask)) {
      *err = "the DIVA solve needs diva with uvel_2d, vvel_2d, btractx, btracty, thck and ice_plus_land_mask";
      return false;
    }
    if (diva) p->diva_io.push_back(*I.diva);
    if (I.nhalo != 2) { *err = "nhalo must be 2"; return false; }
    if (I.nx < 6 || I.ny < 6) { *err = "grid too small"; return false; }
    if (I.pcg_variant != in[0].pcg_variant || I.pcg_ncheck != in[0].pcg_ncheck ||
        I.precision != in[0].precision) {
      *err = "all instances of a batch must share pcg_variant, pcg_ncheck and precision";
      return false;
    }
    if (!I.stagusrf || !I.stagthck || !I.flwafact || !I.active_cell || !I.active_vertex ||
        !I.loadu || !I.loadv || !I.umask_dirichlet || !I.vmask_dirichlet || !I.sigma ||
        (!I.beta_internal && !I.sliding)) {
      *err = "missing input array";
      return false;
    }
    if (I.which_efvs < 0 || I.which_efvs > 2 || I.which_assemble_beta < 0 || I.which_assemble_beta > 1 ||
        I.which_resid < 0 || I.which_resid > 4 || (I.pcg_variant != 2 && I.pcg_variant != 3) ||
        I.which_precond < 0 || I.which_precond > 2 || I.precision < 0 || I.precision > 1 ||
        I.maxiter_nonlinear < 1 || I.pcg_maxiters < 1) {
      *err = "option out of range (which_efvs 0-2, which_assemble_beta 0-1, which_resid 0-4, "
             "pcg_variant 2-3, which_precond 0-2, precision 0-1, iteration caps >= 1)";
      return false;
    }
    if (I.sliding) {
      SlideParams sp;
      if (!slide_params(*I.sliding, &sp, err)) return false;
      if (I.which_babc != I.sliding->law) {
        *err = "which_babc must equal the sliding law";
        return false;
      }
      p->any_sliding = true;
    }
    if (I.guess_mode != BP_GUESS_GIVEN && (I.guess_mode != BP_GUESS_LEARNED || solve2d)) {
      *err = "guess_mode must be BP_GUESS_GIVEN, or BP_GUESS_LEARNED for the 3-D solve";
      return false;
    }
    p->guess_mode.push_back(I.guess_mode);
    p->nx.push_back(I.nx); p->ny.push_back(I.ny); p->periodic.push_back(I.periodic);
    add_columns(I.nx, I.ny, nz, I.periodic, I.active_vertex, b, p, &cms[b], &cols[b]);
    p->ncols += (int)cols[b].size();
  }
  // global columns
  const int NC = p->ncols;
  p->nnodes = NC * nz;
  int nblocks = 0;
  for (int b = 0; b < n; ++b) nblocks += ((int)cols[b].size() + p->W - 1) / p->W;
  p->npad = round_up(std::max(nblocks * p->W * nz, 1), 64);
  p->col_node.assign(NC, 0);
  p->col_h.resize(NC);
  p->col_inst.resize(NC);
  p->col_ij.resize(2 * (size_t)NC);
  p->col_nbr.resize(9 * (size_t)NC);
  p->col_cells.assign(4 * (size_t)NC, -1);
  p->col_beta.resize(NC);
  if (p->any_sliding) p->col_slide.assign(3 * (size_t)NC, 0.0);
  p->load.assign(p->npad, double2{0.0, 0.0});
  p->dmask.assign(p->npad, 0);
  // cells: count first (cell ids must be global)
  std::vector<std::vector<int>> cellid(n);
  for (int b = 0; b < n; ++b) {
    const bp_inputs& I = in[b];
    const int nx = I.nx, ny = I.ny, nh = I.nhalo;
    cellid[b].assign((size_t)nx * ny, -1);
    for (int j = nh + 1; j <= ny - nh + 1; ++j)
      for (int i = nh + 1; i <= nx - nh + 1; ++i)
        if (I.active_cell[cel(i, j, nx)]) {
          cellid[b][cel(i, j, nx)] = p->ncells + (int)cells[b].size();
          cells[b].push_back({i, j});
        }
    p->ncells += (int)cells[b].size();
  }
  const int NCELL = p->ncells;
  p->nelem = solve2d ? NCELL : NCELL * (nz - 1);  // 2-D: one element per cell
  p->nefvs = (l1l2 || diva) ? NCELL * nl : p->nelem;
  p->cell_inst.resize(NCELL);
  p->cell_ij.resize(2 * (size_t)NCELL);
  p->cell_cols.resize(4 * (size_t)NCELL);
  p->cell_s.resize(4 * (size_t)NCELL);
  p->cell_h.resize(4 * (size_t)NCELL);
  p->cell_beta.resize(4 * (size_t)NCELL);
  const bool ssa = solve2d && !l1l2 && !diva;
  p->flwafact.resize((size_t)(ssa ? NCELL : NCELL * nl));
  if (ssa) p->flwafact_layers.resize((size_t)NCELL * nl);
  if (diva) {
    p->cell_thck.resize(NCELL);
    p->eq3_0.resize((size_t)NCELL * 4 * nl);
    p->x2d_0.resize(NC);
    p->col_bt0.resize(NC);
    p->col_ipl.resize(NC);
  }
  if (l1l2) {
    p->cell_flwa.resize((size_t)NCELL * nl);
    p->cell_thck.resize(NCELL);
    p->cell_ds.resize(8 * (size_t)NCELL);
    p->col_ds.resize(2 * (size_t)NC);
  }
  int col_base = 0, cell_base = 0;
  for (int b = 0; b < n; ++b) {
    const bp_inputs& I = in[b];
    const int nx = I.nx, ny = I.ny;
    InstParams& ip = p->inst[b];
    std::memset(&ip, 0, sizeof(ip));
    ip.dx = I.dx; ip.dy = I.dy;
    ip.efvs_constant = I.efvs_constant;
    ip.pcg_tol = I.pcg_tol;
    ip.inner_tol = I.inner_tol > 0.0 ? I.inner_tol : 1.0e-4;
    for (int k = 0; k < nz_in; ++k) ip.sigma[k] = I.sigma[k];
    ip.which_efvs = I.which_efvs;
    ip.which_babc = I.which_babc;
    ip.which_assemble_beta = I.which_assemble_beta;
    ip.which_resid = I.which_resid;
    ip.precond = I.which_precond;
    ip.variant = I.pcg_variant;
    ip.precision = I.precision;
    ip.pcg_maxiters = I.pcg_maxiters;
    ip.ncheck = I.pcg_ncheck > 0 ? I.pcg_ncheck : 5;
    ip.maxiter_nonlinear = I.maxiter_nonlinear;
    if (I.sliding) slide_params(*I.sliding, &ip.slide, err);
    if (l1l2) {
      ip.rhoi = I.l1l2->rhoi;
      ip.grav = I.l1l2->grav;
    }
    const int nc = (int)cols[b].size();
    ip.col_begin = col_base; ip.col_end = col_base + nc;
    add_tiles(p, b, col_base, nc);
    const int ncl = (int)cells[b].size();
    ip.cell_begin = cell_base; ip.cell_end = cell_base + ncl;
    const int epc = solve2d ? 1 : nz - 1;  // elements per cell
    ip.elem_begin = cell_base * epc; ip.elem_end = (cell_base + ncl) * epc;
    for (int c = 0; c < nc; ++c) {
      const int g = col_base + c;
      const int i = cols[b][c].first, j = cols[b][c].second;
      p->col_inst[g] = b;
      p->col_ij[g] = i;
      p->col_ij[NC + g] = j;
      p->col_h[g] = I.stagthck[vtx(i, j, nx)];
      for (int jA = -1; jA <= 1; ++jA)
        for (int iA = -1; iA <= 1; ++iA)
          p->col_nbr[(size_t)((jA + 1) * 3 + (iA + 1)) * NC + g] = cms[b].lookup(i + iA, j + jA);
      // cells (i,j), (i+1,j), (i,j+1), (i+1,j+1): the reference's element order
      const int ci[4] = {i, i + 1, i, i + 1}, cj[4] = {j, j, j + 1, j + 1};
      for (int q = 0; q < 4; ++q) {
        int id = -1;
        if (ci[q] >= 1 && ci[q] <= nx && cj[q] >= 1 && cj[q] <= ny)
          id = cellid[b][cel(ci[q], cj[q], nx)];
        p->col_cells[(size_t)q * NC + g] = id;
      }
      if (I.sliding) {  // recomputed on the device at every Picard iteration
        p->col_beta[g] = 0.0;
        p->col_slide[g] = I.sliding->f_ground[vtx(i, j, nx)];
        slide_vertex(*I.sliding, i, j, nx, &p->col_slide[(size_t)NC + g], &p->col_slide[2 * (size_t)NC + g]);
      } else {
        p->col_beta[g] = I.beta_internal[vtx(i, j, nx)];
      }
      if (diva) {
        const size_t w = vtx(i, j, nx);
        p->x2d_0[g] = double2{I.diva->uvel_2d[w], I.diva->vvel_2d[w]};
        p->col_bt0[g] = double2{I.diva->btractx[w], I.diva->btracty[w]};
        uint8_t bits = 0;
        for (int q = 0; q < 4; ++q)
          if (ci[q] >= 1 && ci[q] <= nx && cj[q] >= 1 && cj[q] <= ny &&
              I.diva->ice_plus_land_mask[cel(ci[q], cj[q], nx)] == 1)
            bits |= (uint8_t)(1u << q);
        p->col_ipl[g] = bits;
      }
      if (l1l2) {
        p->col_ds[g] = I.l1l2->dusrf_dx[vtx(i, j, nx)];
        p->col_ds[(size_t)NC + g] = I.l1l2->dusrf_dy[vtx(i, j, nx)];
      }
      if (solve2d) {
        // load summed over the levels (:2123-2137); the bed level's
        // Dirichlet masks (:2878)
        double lu = 0.0, lv = 0.0;
        for (int k = 0; k < nz_in; ++k) {
          lu = lu + I.loadu[vtx(i, j, nx) * nz_in + k];
          lv = lv + I.loadv[vtx(i, j, nx) * nz_in + k];
        }
        p->load[p->col_node[g]] = double2{lu, lv};
        const size_t bed = vtx(i, j, nx) * nz_in + (nz_in - 1);
        p->dmask[p->col_node[g]] = (uint8_t)((I.umask_dirichlet[bed] == 1 ? 1 : 0) | (I.vmask_dirichlet[bed] == 1 ? 2 : 0));
      } else {
        for (int k = 0; k < nz; ++k) {
          const size_t src = vtx(i, j, nx) * nz + k;
          p->load[node_of(*p, g, k)] = double2{I.loadu[src], I.loadv[src]};
          p->dmask[node_of(*p, g, k)] =
              (uint8_t)((I.umask_dirichlet[src] == 1 ? 1 : 0) | (I.vmask_dirichlet[src] == 1 ? 2 : 0));
        }
      }
    }
    for (int c = 0; c < ncl; ++c) {
      const int g = cell_base + c;
      const int ic = cells[b][c].first, jc = cells[b][c].second;
      p->cell_inst[g] = b;
      p->cell_ij[g] = ic;
      p->cell_ij[NCELL + g] = jc;
      const int vi[4] = {ic - 1, ic, ic, ic - 1}, vj[4] = {jc - 1, jc - 1, jc, jc};
      for (int q = 0; q < 4; ++q) {
        const size_t v = vtx(vi[q], vj[q], nx);
        p->cell_cols[(size_t)q * NCELL + g] = cms[b].lookup(vi[q], vj[q]);
        p->cell_s[(size_t)q * NCELL + g] = I.stagusrf[v];
        p->cell_h[(size_t)q * NCELL + g] = I.stagthck[v];
        p->cell_beta[(size_t)q * NCELL + g] = I.sliding ? 0.0 : I.beta_internal[v];
        if (l1l2) {
          p->cell_ds[(size_t)q * NCELL + g] = I.l1l2->dusrf_dx[v];
          p->cell_ds[(size_t)(4 + q) * NCELL + g] = I.l1l2->dusrf_dy[v];
        }
      }
      if (l1l2) {
        p->cell_thck[g] = I.l1l2->thck[cel(ic, jc, nx)];
        for (int k = 0; k < nl; ++k) p->cell_flwa[(size_t)g * nl + k] = I.l1l2->flwa[cel(ic, jc, nx) * nl + k];
      }
      if (diva) {  // efvs_qp_3d starts from the last solve's efvs on every point (:1166-1170)
        p->cell_thck[g] = I.diva->thck[cel(ic, jc, nx)];
        for (int q = 0; q < 4; ++q)
          for (int k = 0; k < nl; ++k)
            p->eq3_0[((size_t)g * 4 + q) * nl + k] = I.diva->efvs ? I.diva->efvs[cel(ic, jc, nx) * nl + k] : 0.0;
      }
      if (ssa) {
        for (int k = 0; k < nl; ++k)
          p->flwafact_layers[(size_t)g * nl + k] = I.flwafact[cel(ic, jc, nx) * nl + k];
      }
      if (ssa) {  // glissade_vertical_average (glissade_grid_operators.F90:1172-1236)
        double f = 0.0;
        for (int k = 0; k < nz_in - 1; ++k)
          f = f + I.flwafact[cel(ic, jc, nx) * (nz_in - 1) + k] * (I.sigma[k + 1] - I.sigma[k]);
        p->flwafact[g] = f;
      } else {  // per layer (3-D elements; the L1L2 layer viscosities)
        for (int k = 0; k < nl; ++k)
          p->flwafact[(size_t)g * nl + k] = I.flwafact[cel(ic, jc, nx) * nl + k];
      }
    }
    col_base += nc;
    cell_base += ncl;
  }
  fill_nbn(p);
  p->ntiles = (int)p->tile_start.size();
  return true;
}

void gather_velocity(const HostPlan& p, int b, const double* uvel,
                     const double* vvel, double2* x) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], nz = p.nz, NC = p.ncols;
  for (int g = ip.col_begin; g < ip.col_end; ++g) {
    const int i = p.col_ij[g], j = p.col_ij[NC + g];
    if (p.diva) {  // the carried-over mean velocity (:1173-1180)
      x[p.col_node[g]] = p.x2d_0[g];
      continue;
    }
    if (p.solve2d) {  // uvel_2d = uvel(nz,:,:) (glissade_velo_higher.F90:1179-1180)
      const size_t src = vtx(i, j, nx) * p.nz_out + (p.nz_out - 1);
      x[p.col_node[g]] = double2{uvel[src], vvel[src]};
      continue;
    }
    for (int k = 0; k < nz; ++k) {
      const size_t src = vtx(i, j, nx) * nz + k;
      x[node_of(p, g, k)] = double2{uvel[src], vvel[src]};
    }
  }
}

void scatter_vector(const HostPlan& p, int b, const double2* x, double* vu,
                    double* vv) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], nz = p.nz, NC = p.ncols;
  for (int g = ip.col_begin; g < ip.col_end; ++g) {
    const int i = p.col_ij[g], j = p.col_ij[NC + g];
    for (int k = 0; k < nz; ++k) {
      const size_t dst = vtx(i, j, nx) * nz + k;
      const double2 v = x[node_of(p, g, k)];
      if (vu) vu[dst] = v.x;
      if (vv) vv[dst] = v.y;
    }
  }
}

void scatter_velocity(const HostPlan& p, int b, const double2* x,
                      double* uvel, double* vvel) {
  if (p.solve2d) {  // the 2-D velocity on every level (:3745-3750)
    const InstParams& ip = p.inst[b];
    const int nx = p.nx[b], NC = p.ncols, L = p.nz_out;
    for (int g = ip.col_begin; g < ip.col_end; ++g) {
      const size_t w = vtx(p.col_ij[g], p.col_ij[NC + g], nx);
      const double2 xg = x[p.col_node[g]];
      for (int k = 0; k < L; ++k) {
        uvel[w * L + k] = xg.x;
        vvel[w * L + k] = xg.y;
      }
    }
  } else {
    scatter_vector(p, b, x, uvel, vvel);
  }
  halo_stag(p.nx[b], p.ny[b], p.nz_out, p.periodic[b], uvel);
  halo_stag(p.nx[b], p.ny[b], p.nz_out, p.periodic[b], vvel);
}

void scatter_velocity_3d(const HostPlan& p, int b, const double2* x3,
                         double* uvel, double* vvel) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], ny = p.ny[b], NC = p.ncols, L = p.nz_out;
  const size_t nvert = (size_t)(nx - 1) * (ny - 1);
  for (size_t w = 0; w < nvert; ++w)
    for (int k = 0; k < L - 1; ++k) uvel[w * L + k] = vvel[w * L + k] = 0.0;
  for (int g = ip.col_begin; g < ip.col_end; ++g) {
    const size_t w = vtx(p.col_ij[g], p.col_ij[NC + g], nx);
    for (int k = 0; k < L; ++k) {
      uvel[w * L + k] = x3[(size_t)g * L + k].x;
      vvel[w * L + k] = x3[(size_t)g * L + k].y;
    }
  }
  halo_stag(nx, ny, L, p.periodic[b], uvel);
  halo_stag(nx, ny, L, p.periodic[b], vvel);
}

void gather_velocity_3d(const HostPlan& p, int b, const double* uvel,
                        const double* vvel, double2* x3) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], NC = p.ncols, L = p.nz_out;
  for (int g = ip.col_begin; g < ip.col_end; ++g) {
    const size_t w = vtx(p.col_ij[g], p.col_ij[NC + g], nx);
    for (int k = 0; k < L; ++k) x3[(size_t)g * L + k] = double2{uvel[w * L + k], vvel[w * L + k]};
  }
}

void scatter_diva(const HostPlan& p, int b, const double2* x, const double2* bt) {
  const InstParams& ip = p.inst[b];
  const bp_diva& D = p.diva_io[b];
  const int nx = p.nx[b], ny = p.ny[b], NC = p.ncols;
  const size_t nvert = (size_t)(nx - 1) * (ny - 1);
  for (size_t w = 0; w < nvert; ++w) D.uvel_2d[w] = D.vvel_2d[w] = D.btractx[w] = D.btracty[w] = 0.0;
  for (int g = ip.col_begin; g < ip.col_end; ++g) {
    const size_t w = vtx(p.col_ij[g], p.col_ij[NC + g], nx);
    D.uvel_2d[w] = x[p.col_node[g]].x;
    D.vvel_2d[w] = x[p.col_node[g]].y;
    D.btractx[w] = bt[g].x;
    D.btracty[w] = bt[g].y;
  }
  halo_stag(nx, ny, 1, p.periodic[b], D.uvel_2d);
  halo_stag(nx, ny, 1, p.periodic[b], D.vvel_2d);
  halo_stag(nx, ny, 1, p.periodic[b], D.btractx);
  halo_stag(nx, ny, 1, p.periodic[b], D.btracty);
}

void scatter_efvs(const HostPlan& p, int b, const double* efvs_elem,
                  double* efvs) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], ny = p.ny[b], nz = p.nz_out, NCELL = p.ncells;
  std::memset(efvs, 0, sizeof(double) * (size_t)(nz - 1) * nx * ny);
  for (int g = ip.cell_begin; g < ip.cell_end; ++g) {
    const int ic = p.cell_ij[g], jc = p.cell_ij[NCELL + g];
    for (int k = 0; k < nz - 1; ++k)  // shallow-shelf: the cell's value on every layer
      efvs[cel(ic, jc, nx) * (nz - 1) + k] =
          efvs_elem[p.solve2d && !p.l1l2 && !p.diva ? (size_t)g : (size_t)g * (nz - 1) + k];
  }
}

void gather_matrix(const HostPlan& p, const double* Auu, const double* Auv,
                   const double* Avu, const double* Avv, double2* A) {
  const int nx = p.nx[0], nz = p.nz, NC = p.ncols, np = p.npad;
  std::memset((void*)A, 0, sizeof(double2) * 2 * 27 * (size_t)np);
  for (int g = 0; g < NC; ++g) {
    const int i = p.col_ij[g], j = p.col_ij[NC + g];
    for (int k = 0; k < nz; ++k) {
      const size_t n = node_of(p, g, k);
      const size_t base = (vtx(i, j, nx) * nz + k) * 27;
      for (int m = 0; m < 27; ++m) {
        A[(size_t)m * np + n] = double2{Auu[base + m], Auv[base + m]};
        A[(size_t)(27 + m) * np + n] = double2{Avu[base + m], Avv[base + m]};
      }
    }
  }
}

void scatter_matrix(const HostPlan& p, const double2* A, double* Auu,
                    double* Auv, double* Avu, double* Avv) {
  const int nx = p.nx[0], ny = p.ny[0], nz = p.nz, NC = p.ncols, np = p.npad;
  const size_t tot = (size_t)27 * nz * (nx - 1) * (ny - 1);
  for (double* a : {Auu, Auv, Avu, Avv})
    if (a) std::memset(a, 0, sizeof(double) * tot);
  for (int g = 0; g < NC; ++g) {
    const int i = p.col_ij[g], j = p.col_ij[NC + g];
    for (int k = 0; k < nz; ++k) {
      const size_t n = node_of(p, g, k);
      const size_t base = (vtx(i, j, nx) * nz + k) * 27;
      for (int m = 0; m < 27; ++m) {
        const double2 u = A[(size_t)m * np + n], v = A[(size_t)(27 + m) * np + n];
        if (Auu) Auu[base + m] = u.x;
        if (Auv) Auv[base + m] = u.y;
        if (Avu) Avu[base + m] = v.x;
        if (Avv) Avv[base + m] = v.y;
      }
    }
  }
}

void scatter_matrix_sym(const HostPlan& p, const double2* A, double* Auu,
                        double* Auv, double* Avu, double* Avv) {
  const int nx = p.nx[0], ny = p.ny[0], nz = p.nz, NC = p.ncols, np = p.npad;
  const size_t tot = (size_t)27 * nz * (nx - 1) * (ny - 1);
  for (double* a : {Auu, Auv, Avu, Avv})
    if (a) std::memset(a, 0, sizeof(double) * tot);
  for (int g = 0; g < NC; ++g) {
    const int i = p.col_ij[g], j = p.col_ij[NC + g];
    for (int k = 0; k < nz; ++k) {
      const size_t n = node_of(p, g, k);
      const size_t base = (vtx(i, j, nx) * nz + k) * 27;
      for (int m = 0; m < 27; ++m) {
        double uu, uv, vu, vv;
        if (m >= 13) {
          const double2 a0 = A[(size_t)(m - 13) * np + n], a1 = A[(size_t)(14 + m - 13) * np + n];
          uu = a0.x; uv = a0.y; vu = a1.x; vv = a1.y;
        } else {
          const int iA = m % 3 - 1, jA = (m / 3) % 3 - 1, kA = m / 9 - 1;
          const int cn = p.col_nbr[(size_t)((jA + 1) * 3 + (iA + 1)) * NC + g];
          const int kn = k + kA;
          if (cn < 0 || kn < 0 || kn >= nz) continue;
          const size_t pn = node_of(p, cn, kn);
          const double2 b0 = A[(size_t)(13 - m) * np + pn], b1 = A[(size_t)(14 + 13 - m) * np + pn];
          uu = b0.x; uv = b1.x; vu = b0.y; vv = b1.y;
        }
        if (Auu) Auu[base + m] = uu;
        if (Auv) Auv[base + m] = uv;
        if (Avu) Avu[base + m] = vu;
        if (Avv) Avv[base + m] = vv;
      }
    }
  }
}

void gather_matrix_sym(const HostPlan& p, const double* Auu, const double* Auv,
                       const double* Avu, const double* Avv, double2* A) {
  const int nx = p.nx[0], nz = p.nz, NC = p.ncols, np = p.npad;
  std::memset((void*)A, 0, sizeof(double2) * 2 * 14 * (size_t)np);
  for (int g = 0; g < NC; ++g) {
    const int i = p.col_ij[g], j = p.col_ij[NC + g];
    for (int k = 0; k < nz; ++k) {
      const size_t n = node_of(p, g, k);
      const size_t base = (vtx(i, j, nx) * nz + k) * 27;
      for (int m = 13; m < 27; ++m) {
        A[(size_t)(m - 13) * np + n] = double2{Auu[base + m], Auv[base + m]};
        A[(size_t)(14 + m - 13) * np + n] = double2{Avu[base + m], Avv[base + m]};
      }
    }
  }
}

void halo_cells(int nx, int ny, int periodic, double* a) {
  auto at = [&](int i, int j) -> double& { return a[cel(i, j, nx)]; };
  if (!periodic) {
    for (int j = 3; j <= ny - 2; ++j) at(1, j) = at(2, j) = at(nx - 1, j) = at(nx, j) = 0.0;
    for (int i = 1; i <= nx; ++i) at(i, 1) = at(i, 2) = at(i, ny - 1) = at(i, ny) = 0.0;
    return;
  }
  for (int j = 3; j <= ny - 2; ++j) {
    const double e1 = at(nx - 3, j), e2 = at(nx - 2, j), w1 = at(3, j), w2 = at(4, j);
    at(1, j) = e1; at(2, j) = e2; at(nx - 1, j) = w1; at(nx, j) = w2;
  }
  for (int i = 1; i <= nx; ++i) {
    const double n1 = at(i, ny - 3), n2 = at(i, ny - 2), s1 = at(i, 3), s2 = at(i, 4);
    at(i, 1) = n1; at(i, 2) = n2; at(i, ny - 1) = s1; at(i, ny) = s2;
  }
}

void scatter_elements(const HostPlan& p, int b, const double* vals, int nv,
                      double* const* out) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], ny = p.ny[b], nz = p.nz_out, NCELL = p.ncells;
  const size_t ne = (size_t)diagnostic_elements(p);
  for (int f = 0; f < nv; ++f) {
    if (!out[f]) continue;
    std::memset(out[f], 0, sizeof(double) * (size_t)(nz - 1) * nx * ny);
    for (int g = ip.cell_begin; g < ip.cell_end; ++g) {
      const int ic = p.cell_ij[g], jc = p.cell_ij[NCELL + g];
      for (int k = 0; k < nz - 1; ++k)
        out[f][cel(ic, jc, nx) * (nz - 1) + k] = vals[(size_t)f * ne + (size_t)g * (nz - 1) + k];
    }
  }
}

DevView diagnostics_view(const DevView& v, const HostPlan& p, double2* x3, const double* flwafact_layers,
                         const int* col_node3) {
  if (!p.solve2d) return v;
  DevView d = v;
  d.nz = p.nz_out;
  d.nelem = diagnostic_elements(p);
  d.x = x3;  // [ncols][nz_out]: node (col, k) = col * nz_out + k
  d.W = 1;
  d.lsh = 0;
  d.col_node = col_node3;
  if (!p.l1l2 && !p.diva) d.flwafact = flwafact_layers;
  return d;
}

void scatter_bfric(const HostPlan& p, int b, int which, const double* vals,
                   double* bfricflx) {
  const InstParams& ip = p.inst[b];
  const int nx = p.nx[b], ny = p.ny[b], NCELL = p.ncells, NC = p.ncols;
  std::memset(bfricflx, 0, sizeof(double) * (size_t)nx * ny);
  if (which == 0) {
    for (int g = ip.cell_begin; g < ip.cell_end; ++g)
      bfricflx[cel(p.cell_ij[g], p.cell_ij[NCELL + g], nx)] = vals[g];
  } else {
    // vertex values at the owned active vertices, halo vertices from their
    // images; cells next to the halo are overwritten by the halo update
    std::vector<double> st((size_t)(nx - 1) * (ny - 1), 0.0);
    for (int g = ip.col_begin; g < ip.col_end; ++g) st[vtx(p.col_ij[g], p.col_ij[NC + g], nx)] = vals[g];
    halo_stag(nx, ny, 1, p.periodic[b], st.data());
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        bfricflx[cel(i, j, nx)] = (st[vtx(i, j, nx)] + st[vtx(i - 1, j, nx)] + st[vtx(i, j - 1, nx)] +
                                   st[vtx(i - 1, j - 1, nx)]) / 4.0;
  }
  halo_cells(nx, ny, p.periodic[b], bfricflx);
}

void halo_stag(int nx, int ny, int nlead, int periodic, double* a) {
  const int V = nx - 1, W = ny - 1;
  auto at = [&](int l, int i, int j) -> double& {
    return a[((size_t)(j - 1) * V + (i - 1)) * nlead + l];
  };
  if (!periodic) {
    for (int j = 1; j <= W; ++j)
      for (int l = 0; l < nlead; ++l) { at(l, 1, j) = 0.0; at(l, V, j) = 0.0; }
    for (int i = 1; i <= V; ++i)
      for (int l = 0; l < nlead; ++l) { at(l, i, 1) = 0.0; at(l, i, W) = 0.0; }
    return;
  }
  for (int j = 3; j <= W - 1; ++j)
    for (int l = 0; l < nlead; ++l) {
      const double w = at(l, 3, j), e1 = at(l, V - 2, j), e2 = at(l, V - 1, j);
      at(l, V, j) = w; at(l, 1, j) = e1; at(l, 2, j) = e2;
    }
  for (int i = 1; i <= V; ++i)
    for (int l = 0; l < nlead; ++l) {
      const double s = at(l, i, 3), n1 = at(l, i, W - 2), n2 = at(l, i, W - 1);
      at(l, i, W) = s; at(l, i, 1) = n1; at(l, i, 2) = n2;
    }
}

}  // namespace bp
