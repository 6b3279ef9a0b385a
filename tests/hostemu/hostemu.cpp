// hostemu.cpp -- TEST ONLY.  Runs the device kernels' per-thread bodies
// (cism_b200/csrc/bp_body.h) sequentially on the CPU through the same host
// plan, so the compaction, periodic images and assembly indexing can be
// checked against the oracle without a GPU.  Not part of the product
// library and never loaded by it.
#include <cstring>
#include <string>
#include <vector>

#include "bp_body.h"
#include "bp_oracle.h"
#include "bp_plan.h"

using namespace bp;

namespace {
struct Emu {
  HostPlan p;
  std::vector<InstParams> inst;
  std::vector<InstState> st;
  std::vector<double> qp, efvs, badj, lw, eq3, omk, om, somega, beff;
  std::vector<double2> A, x, b, x3, bt;
  DevView v;
  void bind() {
    std::memset(&v, 0, sizeof(v));
    v.nz = p.nz; v.ncols = p.ncols; v.nnodes = p.nnodes; v.npad = p.npad;
    v.W = p.W; v.lsh = p.lsh;
    v.tile_threads = std::min(kTile, (p.W * p.nz + 31) / 32 * 32);
    v.col_node = p.col_node.data(); v.col_nbn = p.col_nbn.data();
    v.tile_start = p.tile_start.data(); v.tile_end = p.tile_end.data(); v.tile_inst = p.tile_inst.data();
    v.tile_ncols = p.tile_ncols.data(); v.tile_col0 = p.tile_col0.data();
    v.solve2d = p.solve2d ? 1 : 0;
    v.l1l2 = p.l1l2 ? 1 : 0;
    v.diva = p.diva ? 1 : 0;
    v.nl = p.nz_out - 1;
    v.ncells = p.ncells; v.nelem = p.nelem; v.ninst = p.ninst; v.ntiles = p.ntiles;
    int anyd = 0;
    for (auto m : p.dmask) anyd |= m != 0;
    v.any_dirichlet = anyd;
    v.inst = p.inst.data();
    st.assign(p.ninst, InstState{});
    v.st = st.data();
    v.col_inst = p.col_inst.data(); v.col_nbr = p.col_nbr.data(); v.col_cells = p.col_cells.data();
    v.col_ij = p.col_ij.data(); v.col_beta = p.col_beta.data(); v.load = p.load.data();
    v.dmask = p.dmask.data(); v.cell_inst = p.cell_inst.data(); v.cell_ij = p.cell_ij.data();
    v.cell_cols = p.cell_cols.data(); v.cell_s = p.cell_s.data(); v.cell_h = p.cell_h.data();
    v.cell_beta = p.cell_beta.data(); v.flwafact = p.flwafact.data();
    qp.assign((size_t)p.nelem * 80, 0.0); v.qp = qp.data();
    efvs.assign(std::max(p.nefvs, 1), 0.0); v.efvs = efvs.data();
    if (p.l1l2) {
      v.cell_flwa = p.cell_flwa.data(); v.cell_thck = p.cell_thck.data(); v.cell_ds = p.cell_ds.data();
      v.col_ds = p.col_ds.data(); v.col_h = p.col_h.data();
      lw.assign(4 * (size_t)v.nl * std::max(p.ncells, 1), 0.0); v.lw = lw.data();
      x3.assign((size_t)std::max(p.ncols, 1) * (v.nl + 1), double2{0, 0}); v.x3 = x3.data();
    }
    if (p.diva) {
      const size_t nc = (size_t)std::max(p.ncells, 1), ncol = (size_t)std::max(p.ncols, 1);
      v.cell_thck = p.cell_thck.data(); v.col_ipl = p.col_ipl.data();
      eq3 = p.eq3_0; eq3.resize(std::max<size_t>(eq3.size(), 1)); v.eq3 = eq3.data();
      omk.assign(nc * (v.nl + 1), 0.0); v.cell_omk = omk.data();
      om.assign(nc, 0.0); v.cell_om = om.data();
      somega.assign(ncol, 0.0); v.col_somega = somega.data();
      beff.assign(ncol, 0.0); v.col_beff = beff.data();
      bt = p.col_bt0; bt.resize(ncol); v.col_bt = bt.data();
      x3.assign(ncol * (v.nl + 1), double2{0, 0}); v.x3 = x3.data();
    }
    badj.assign(4 * (size_t)p.npad, 0.0); v.badj = badj.data();
    A.assign(2 * 27 * (size_t)p.npad, double2{0, 0}); v.A = A.data();
    x.assign(p.npad, double2{0, 0}); v.x = x.data();
    b.assign(p.npad, double2{0, 0}); v.b = b.data();
  }
};

// Every node (n, col, k) of a plan, column by column (the engine's layout:
// node_of).
template <typename F>
void each_node(const HostPlan& p, F f) {
  for (int c = 0; c < p.ncols; ++c)
    for (int k = 0; k < p.nz; ++k) f(node_of(p, c, k), c, k);
}

// Ke: the element blocks of the element-centric form (row_gather), or
// null for the row-integrating form (row_assemble).
template <int B>
void rows(Emu& E, const RefTables& T, const double* Ke) {
  const DevView& v = E.v;
  double* Ad = reinterpret_cast<double*>(E.A.data());
  each_node(E.p, [&](size_t n, int col, int k) {
    double acc[27];
    if (Ke) row_gather<B>(v, Ke, col, k, acc);
    else row_assemble<B>(v, T, col, k, acc);
    row_basal<B>(v, T, col, k, acc);
    const double adj = row_dirichlet<B>(v, col, k, acc);
    for (int m = 0; m < 27; ++m)
      Ad[(((size_t)((B >> 1) * 27 + m)) * v.npad + n) * 2 + (B & 1)] = acc[m];
    E.badj[(size_t)B * v.npad + n] = adj;
  });
}
}  // namespace

// gather = 1: pass 2 in the element-centric form (element_row_blocks for
// every element and corner, then row_gather), as k_asm_elem + k_asm_rows.
extern "C" int emu_assemble_form(const bp_inputs* in, const double* uvel, const double* vvel,
                                 double* Auu, double* Auv, double* Avu, double* Avv, double* bu,
                                 double* bv, double* efvs, int gather) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err)) return 10;
  E.bind();
  gather_velocity(E.p, 0, uvel, vvel, E.x.data());
  RefTables T;
  fill_ref_tables(&T);
  for (int e = 0; e < E.p.nelem; ++e) {
    double s = 0.0;
    for (int p = 0; p < 8; ++p) {
      double out[10], eq = 0.0;
      if (!qp_element_point(E.v, T, e, p, out, &eq)) return 2;
      std::memcpy(&E.qp[((size_t)e * 8 + p) * 10], out, sizeof(out));
      s += eq;
    }
    E.efvs[e] = s / 8.0;
  }
  std::vector<double> Ke;
  if (gather) {
    Ke.assign((size_t)E.p.nelem * 256, 0.0);
    for (int e = 0; e < E.p.nelem; ++e)
      for (int nr = 0; nr < 8; ++nr) {
        double K[32];
        element_row_blocks(T, &E.qp[(size_t)e * 80], nr, K);
        for (int b = 0; b < 4; ++b)
          for (int nc = 0; nc < 8; ++nc) Ke[(size_t)e * 256 + b * 64 + nr * 8 + nc] = K[b * 8 + nc];
      }
  }
  const double* ke = gather ? Ke.data() : nullptr;
  rows<0>(E, T, ke); rows<1>(E, T, ke); rows<2>(E, T, ke); rows<3>(E, T, ke);
  const size_t np = E.p.npad;
  for (int n = 0; n < E.p.npad; ++n) {  // the hole slots are zero
    const uint8_t dm = E.p.dmask[n];
    double u = E.p.load[n].x - E.badj[n] - E.badj[np + n];
    double w = E.p.load[n].y - E.badj[2 * np + n] - E.badj[3 * np + n];
    if (dm & 1) u = E.x[n].x;
    if (dm & 2) w = E.x[n].y;
    E.b[n] = double2{u, w};
  }
  scatter_matrix(E.p, E.A.data(), Auu, Auv, Avu, Avv);
  const size_t tot = (size_t)in->nz * (in->nx - 1) * (in->ny - 1);
  std::memset(bu, 0, tot * 8);
  std::memset(bv, 0, tot * 8);
  scatter_vector(E.p, 0, E.b.data(), bu, bv);
  scatter_efvs(E.p, 0, E.efvs.data(), efvs);
  return 0;
}

extern "C" int emu_assemble(const bp_inputs* in, const double* uvel, const double* vvel,
                            double* Auu, double* Auv, double* Avu, double* Avv, double* bu,
                            double* bv, double* efvs) {
  return emu_assemble_form(in, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv, efvs, 0);
}

// Symmetric storage (14 upper offsets; fp32 = 1 for the packed FP32 copy).
extern "C" int emu_matvec_sym(int nx, int ny, int nz, int periodic, const int* active_vertex,
                              const double* Auu, const double* Auv, const double* Avu,
                              const double* Avv, const double* xu, const double* xv, double* yu,
                              double* yv, int fp32) {
  Emu E;
  std::string err;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &E.p, &err)) return 10;
  E.bind();
  E.v.sym = 1;
  std::vector<double2> As(2 * 14 * (size_t)E.p.npad);
  gather_matrix_sym(E.p, Auu, Auv, Avu, Avv, As.data());
  std::vector<float4> A32(14 * (size_t)E.p.npad);
  std::vector<double2> A32d(2 * (size_t)E.p.npad);
  E.v.A = As.data();
  E.v.A32 = A32.data();
  E.v.A32d = A32d.data();
  each_node(E.p, [&](size_t n, int col, int k) { make_a32_row(E.v, col, k, n); });
  gather_velocity(E.p, 0, xu, xv, E.x.data());
  std::vector<double2> y(E.p.npad, double2{0, 0});
  const double2* xs = E.x.data();
  auto src = [xs](size_t m) { return xs[m]; };
  each_node(E.p, [&](size_t n, int col, int k) {
    y[n] = fp32 ? matvec_row_sym32(E.v, A32.data(), col, k, n, src)
                : matvec_row_sym(E.v, As.data(), col, k, n, src);
  });
  const size_t tot = (size_t)nz * (nx - 1) * (ny - 1);
  std::memset(yu, 0, tot * 8);
  std::memset(yv, 0, tot * 8);
  scatter_vector(E.p, 0, y.data(), yu, yv);
  return 0;
}

extern "C" int emu_matvec(int nx, int ny, int nz, int periodic, const int* active_vertex,
                          const double* Auu, const double* Auv, const double* Avu,
                          const double* Avv, const double* xu, const double* xv, double* yu,
                          double* yv) {
  Emu E;
  std::string err;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &E.p, &err)) return 10;
  E.bind();
  gather_matrix(E.p, Auu, Auv, Avu, Avv, E.A.data());
  gather_velocity(E.p, 0, xu, xv, E.x.data());
  std::vector<double2> y(E.p.npad, double2{0, 0});
  const double2* xs = E.x.data();
  auto src = [xs](size_t m) { return xs[m]; };
  each_node(E.p, [&](size_t n, int col, int k) { y[n] = matvec_row(E.v, E.A.data(), col, k, n, src); });
  const size_t tot = (size_t)nz * (nx - 1) * (ny - 1);
  std::memset(yu, 0, tot * 8);
  std::memset(yv, 0, tot * 8);
  scatter_vector(E.p, 0, y.data(), yu, yv);
  return 0;
}

// SIA column preconditioner z = M^-1 r (sym = 1: half storage as solves use;
// 0: full rows as bp_pcg uses), the column loop of the device tile routine.
extern "C" int emu_sia_apply(int nx, int ny, int nz, int periodic, const int* active_vertex,
                             const double* Auu, const double* Auv, const double* Avu,
                             const double* Avv, const double* ru, const double* rv, double* zu,
                             double* zv, int sym) {
  Emu E;
  std::string err;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &E.p, &err)) return 10;
  E.bind();
  std::vector<double2> As;
  if (sym) {
    As.assign(2 * 14 * (size_t)E.p.npad, double2{0, 0});
    gather_matrix_sym(E.p, Auu, Auv, Avu, Avv, As.data());
    E.v.sym = 1;
    E.v.A = As.data();
  } else {
    gather_matrix(E.p, Auu, Auv, Avu, Avv, E.A.data());
  }
  gather_velocity(E.p, 0, ru, rv, E.x.data());
  // the factors of the linear solve (k_sia_factor), then the two sweeps per
  // column and component (sia_tile)
  std::vector<double2> f(3 * (size_t)E.p.npad, double2{0, 0});
  E.v.sia_f = f.data();
  for (int c = 0; c < E.p.ncols; ++c)
    for (int h = 0; h < 2; ++h) sia_factor_column(E.v, c, h);
  std::vector<double> s((size_t)nz);
  std::vector<double2> z(E.p.npad, double2{0, 0});
  for (int c = 0; c < E.p.ncols; ++c) {
    for (int h = 0; h < 2; ++h) {
      for (int k = 0; k < nz; ++k) {
        const size_t n = node_of(E.p, c, k);
        s[k] = h ? E.x[n].y : E.x[n].x;
      }
      sia_solve(E.v, nz, h, [&](int k) { return node_of(E.p, c, k); }, s.data(), 1);
      for (int k = 0; k < nz; ++k) (h ? z[node_of(E.p, c, k)].y : z[node_of(E.p, c, k)].x) = s[k];
    }
  }
  const size_t tot = (size_t)nz * (nx - 1) * (ny - 1);
  std::memset(zu, 0, tot * 8);
  std::memset(zv, 0, tot * 8);
  scatter_vector(E.p, 0, z.data(), zu, zv);
  return 0;
}

// Sliding-law beta of every column from the basal velocity (the per-column
// body of k_slide_beta), written to beta (nx-1,ny-1) at each column's
// vertex; other entries are left as they are.  10 if the plan rejects the
// inputs.
extern "C" int emu_slide_beta(const bp_inputs* in, const double* uvel, const double* vvel,
                              double* beta) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err)) return 10;
  E.bind();
  gather_velocity(E.p, 0, uvel, vvel, E.x.data());
  const int nz = E.p.nz, NC = E.p.ncols, nx = in->nx;
  const SlideParams& sp = E.p.inst[0].slide;
  for (int c = 0; c < NC; ++c) {
    const double2 ub = E.x[node_of(E.p, c, nz - 1)];
    const double b = slide_beta(sp, E.p.col_slide[c], E.p.col_slide[(size_t)NC + c],
                                E.p.col_slide[2 * (size_t)NC + c], ub.x, ub.y);
    const int i = E.p.col_ij[c], j = E.p.col_ij[NC + c];
    beta[(size_t)(j - 1) * (nx - 1) + (i - 1)] = b;
  }
  return 0;
}

// Post-solve diagnostics at velocity (uvel, vvel) through the device's
// per-element and per-cell/column bodies and the engine's scatters: the six
// element stresses (nz-1,nx,ny) and bfricflx (nx,ny) by method which.
// beta (nx-1,ny-1), when given, replaces the plan's betas: each column
// takes its vertex's value, each cell corner its column's (0 without one).
static int diagnostics(const bp_inputs* in, const double* uvel, const double* vvel, const double* efvs,
                       const double* beta, int which, double* tau_xz, double* tau_yz, double* tau_xx,
                       double* tau_yy, double* tau_xy, double* tau_eff, double* bfricflx);

extern "C" int emu_diagnostics(const bp_inputs* in, const double* uvel, const double* vvel,
                               const double* beta, int which, double* tau_xz, double* tau_yz,
                               double* tau_xx, double* tau_yy, double* tau_xy, double* tau_eff,
                               double* bfricflx) {
  return diagnostics(in, uvel, vvel, nullptr, beta, which, tau_xz, tau_yz, tau_xx, tau_yy, tau_xy, tau_eff,
                     bfricflx);
}

// The same for a 2-D solve (shallow-shelf, L1L2, DIVA): the 3-D elements
// over the model's levels with the 3-D velocity (uvel, vvel) through the
// engine's diagnostics view; efvs (nz-1,nx,ny) is the L1L2 layer viscosity.
extern "C" int emu_diagnostics_2d(const bp_inputs* in, const double* uvel, const double* vvel,
                                  const double* efvs, int which, double* tau_xz, double* tau_yz,
                                  double* tau_xx, double* tau_yy, double* tau_xy, double* tau_eff,
                                  double* bfricflx) {
  return diagnostics(in, uvel, vvel, efvs, nullptr, which, tau_xz, tau_yz, tau_xx, tau_yy, tau_xy, tau_eff,
                     bfricflx);
}

static int diagnostics(const bp_inputs* in, const double* uvel, const double* vvel, const double* efvs,
                       const double* beta, int which, double* tau_xz, double* tau_yz, double* tau_xx,
                       double* tau_yy, double* tau_xy, double* tau_eff, double* bfricflx) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err)) return 10;
  const int nx = in->nx, NC = E.p.ncols, NCELL = E.p.ncells;
  if (beta) {
    for (int g = 0; g < NC; ++g)
      E.p.col_beta[g] = beta[(size_t)(E.p.col_ij[NC + g] - 1) * (nx - 1) + (E.p.col_ij[g] - 1)];
    for (int q = 0; q < 4; ++q)
      for (int c = 0; c < NCELL; ++c) {
        const int col = E.p.cell_cols[(size_t)q * NCELL + c];
        E.p.cell_beta[(size_t)q * NCELL + c] = col >= 0 ? E.p.col_beta[col] : 0.0;
      }
  }
  E.bind();
  gather_velocity(E.p, 0, uvel, vvel, E.x.data());
  // a 2-D solve: its 3-D velocity and, for L1L2, its layer viscosities
  std::vector<double2> x3(E.p.solve2d ? (size_t)std::max(NC, 1) * E.p.nz_out : 0);
  if (E.p.solve2d) gather_velocity_3d(E.p, 0, uvel, vvel, x3.data());
  if (E.p.l1l2 && efvs) {
    const int nl = E.v.nl;
    for (int c = 0; c < NCELL; ++c) {
      const size_t cc = (size_t)(E.p.cell_ij[NCELL + c] - 1) * nx + (E.p.cell_ij[c] - 1);
      for (int k = 0; k < nl; ++k) E.efvs[(size_t)c * nl + k] = efvs[cc * nl + k];
    }
  }
  std::vector<int> cn3(std::max(NC, 1));
  for (int c = 0; c < NC; ++c) cn3[c] = c * E.p.nz_out;
  const DevView v = diagnostics_view(E.v, E.p, x3.data(), E.p.flwafact_layers.data(), cn3.data());
  RefTables T;
  fill_ref_tables(&T);
  const size_t ne = (size_t)diagnostic_elements(E.p);
  std::vector<double> tau(6 * ne), bf((size_t)std::max(NCELL, NC));
  for (size_t e = 0; e < ne; ++e) {
    double t[6];
    if (!stress_element(v, T, (int)e, t)) return 2;
    for (int q = 0; q < 6; ++q) tau[(size_t)q * ne + e] = t[q];
  }
  const int n = which == 0 ? NCELL : NC;
  for (int i = 0; i < n; ++i) bf[i] = which == 0 ? bfric_cell(v, T, i) : bfric_vertex(v, i);
  double* outs[6] = {tau_xz, tau_yz, tau_xx, tau_yy, tau_xy, tau_eff};
  scatter_elements(E.p, 0, tau.data(), 6, outs);
  scatter_bfric(E.p, 0, which, bf.data(), bfricflx);
  return 0;
}

// One assembled 2-D system (shallow-shelf or L1L2) at velocity (uvel,
// vvel) (the bed level is the 2-D velocity) through the device's 2-D
// bodies: the matrix in (27,1,nx-1,ny-1) and b (nx-1,ny-1); efvs
// (nz-1,nx,ny).  10 if the plan rejects the inputs or they are not a 2-D
// problem, 2 for a singular Jacobian.
extern "C" int emu_assemble_2d(const bp_inputs* in, const double* uvel, const double* vvel,
                               double* Auu, double* Auv, double* Avu, double* Avv, double* bu,
                               double* bv, double* efvs) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err) || !E.p.solve2d) return 10;
  E.bind();
  gather_velocity(E.p, 0, uvel, vvel, E.x.data());
  RefTables T;
  fill_ref_tables(&T);
  const int nl = E.v.nl;
  for (int c = 0; c < E.p.ncells; ++c) {
    double s = 0.0, sk[kNzMax] = {0.0};
    for (int p = 0; p < 4; ++p) {
      double out[5], eq = 0.0, ek[kNzMax];
      if (!qp2_element_point(E.v, T, c, p, out, &eq, ek)) return 2;
      std::memcpy(&E.qp[((size_t)c * 8 + p) * 10], out, sizeof(out));
      s += eq;
      if (E.p.l1l2)
        for (int k = 0; k < nl; ++k) sk[k] += ek[k];
    }
    if (E.p.l1l2)
      for (int k = 0; k < nl; ++k) E.efvs[(size_t)c * nl + k] = sk[k] / 4.0;
    else
      E.efvs[c] = s / 4.0;
  }
  const DevView& v = E.v;
  double* Ad = reinterpret_cast<double*>(E.A.data());
  for (int B = 0; B < 4; ++B)
    for (int col = 0; col < v.ncols; ++col) {
      const size_t n = (size_t)v.col_node[col];
      double acc[27];
      double adj = 0.0;
      switch (B) {
        case 0: row_assemble2<0>(v, T, col, acc); row_basal<0>(v, T, col, 0, acc); adj = row_dirichlet<0>(v, col, 0, acc); break;
        case 1: row_assemble2<1>(v, T, col, acc); row_basal<1>(v, T, col, 0, acc); adj = row_dirichlet<1>(v, col, 0, acc); break;
        case 2: row_assemble2<2>(v, T, col, acc); row_basal<2>(v, T, col, 0, acc); adj = row_dirichlet<2>(v, col, 0, acc); break;
        default: row_assemble2<3>(v, T, col, acc); row_basal<3>(v, T, col, 0, acc); adj = row_dirichlet<3>(v, col, 0, acc); break;
      }
      for (int m = 0; m < 27; ++m)
        Ad[(((size_t)((B >> 1) * 27 + m)) * v.npad + n) * 2 + (B & 1)] = acc[m];
      E.badj[(size_t)B * v.npad + n] = adj;
    }
  const size_t np = E.p.npad;
  for (int n = 0; n < E.p.npad; ++n) {  // the hole slots are zero
    const uint8_t dm = E.p.dmask[n];
    double u = E.p.load[n].x - E.badj[n] - E.badj[np + n];
    double w = E.p.load[n].y - E.badj[2 * np + n] - E.badj[3 * np + n];
    if (dm & 1) u = E.x[n].x;
    if (dm & 2) w = E.x[n].y;
    E.b[n] = double2{u, w};
  }
  scatter_matrix(E.p, E.A.data(), Auu, Auv, Avu, Avv);
  const size_t tot = (size_t)(in->nx - 1) * (in->ny - 1);
  std::memset(bu, 0, tot * 8);
  std::memset(bv, 0, tot * 8);
  scatter_vector(E.p, 0, E.b.data(), bu, bv);
  scatter_efvs(E.p, 0, E.efvs.data(), efvs);
  return 0;
}

// The L1L2 3-D velocity through the device's reconstruction bodies
// (l1l2_cell over the cells, l1l2_column over the columns) and the host
// scatter: basal velocity from the bed level of (uvel, vvel), layer
// viscosities efvs (nz-1,nx,ny); (uout, vout) (nz,nx-1,ny-1) keep their
// bed level away from the columns.  10 if the plan rejects the inputs or
// they are not an L1L2 problem.
extern "C" int emu_velocity_3d_l1l2(const bp_inputs* in, const double* uvel, const double* vvel,
                                    const double* efvs, double* uout, double* vout) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err) || !E.p.l1l2) return 10;
  E.bind();
  gather_velocity(E.p, 0, uvel, vvel, E.x.data());
  const int nl = E.v.nl, NCELL = E.p.ncells, nx = in->nx;
  for (int c = 0; c < NCELL; ++c) {
    const int ic = E.p.cell_ij[c], jc = E.p.cell_ij[NCELL + c];
    for (int k = 0; k < nl; ++k)
      E.efvs[(size_t)c * nl + k] = efvs[((size_t)(jc - 1) * nx + (ic - 1)) * nl + k];
  }
  for (int c = 0; c < NCELL; ++c) l1l2_cell(E.v, c);
  for (int col = 0; col < E.p.ncols; ++col) l1l2_column(E.v, col);
  scatter_velocity_3d(E.p, 0, E.x3.data(), uout, vout);
  return 0;
}

// One DIVA iteration's device bodies on the host plan, without the linear
// solve: assembly pass 1 with the point viscosities (qp2_element_point,
// diva_point_efvs), the cell integrals, beta_eff, the rows with the basal
// and Dirichlet terms, then the traction and 3-D velocity of the mean
// velocity it started from (diva_column_velocity) and the scatters.  The
// mean velocity, traction and viscosities come from in->diva; outputs:
// the matrix and b as emu_assemble_2d, efvs (nz-1,nx,ny), eq3
// (4*(nz-1),nx,ny), omega_k (nz,nx,ny), omega (nx,ny), beta_eff
// (nx-1,ny-1), the 3-D velocity (uout, vout: their bed level kept away from
// the columns) and in->diva's uvel_2d .. btracty written back.
extern "C" int emu_diva_step(const bp_inputs* in, double* Auu, double* Auv, double* Avu, double* Avv,
                             double* bu, double* bv, double* efvs, double* eq3, double* omega_k,
                             double* omega, double* beta_eff, double* uout, double* vout) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err) || !E.p.diva) return 10;
  E.bind();
  std::vector<double> dummy((size_t)in->nz * (in->nx - 1) * (in->ny - 1), 0.0);
  gather_velocity(E.p, 0, dummy.data(), dummy.data(), E.x.data());
  RefTables T;
  fill_ref_tables(&T);
  const int nl = E.v.nl, NCELL = E.p.ncells, NC = E.p.ncols, nx = in->nx, ny = in->ny;
  for (int c = 0; c < NCELL; ++c) {
    double sk[kNzMax] = {0.0};
    for (int p = 0; p < 4; ++p) {
      double out[5], eq = 0.0, ek[kNzMax];
      if (!qp2_element_point(E.v, T, c, p, out, &eq, ek)) return 2;
      std::memcpy(&E.qp[((size_t)c * 8 + p) * 10], out, sizeof(out));
      for (int k = 0; k < nl; ++k) sk[k] += ek[k];
    }
    for (int k = 0; k < nl; ++k) E.efvs[(size_t)c * nl + k] = sk[k] / 4.0;
  }
  for (int c = 0; c < NCELL; ++c) diva_cell_integrals(E.v, c);
  for (int col = 0; col < NC; ++col) diva_column_beta(E.v, col);
  for (int c = 0; c < NCELL; ++c)
    for (int q = 0; q < 4; ++q) {
      const int col = E.p.cell_cols[(size_t)q * NCELL + c];
      E.p.cell_beta[(size_t)q * NCELL + c] = col >= 0 ? E.beff[col] : 0.0;
    }
  const DevView& v = E.v;
  double* Ad = reinterpret_cast<double*>(E.A.data());
  for (int B = 0; B < 4; ++B)
    for (int col = 0; col < v.ncols; ++col) {
      const size_t n = (size_t)v.col_node[col];
      double acc[27];
      double adj = 0.0;
      switch (B) {
        case 0: row_assemble2<0>(v, T, col, acc); row_basal<0>(v, T, col, 0, acc); adj = row_dirichlet<0>(v, col, 0, acc); break;
        case 1: row_assemble2<1>(v, T, col, acc); row_basal<1>(v, T, col, 0, acc); adj = row_dirichlet<1>(v, col, 0, acc); break;
        case 2: row_assemble2<2>(v, T, col, acc); row_basal<2>(v, T, col, 0, acc); adj = row_dirichlet<2>(v, col, 0, acc); break;
        default: row_assemble2<3>(v, T, col, acc); row_basal<3>(v, T, col, 0, acc); adj = row_dirichlet<3>(v, col, 0, acc); break;
      }
      for (int m = 0; m < 27; ++m)
        Ad[(((size_t)((B >> 1) * 27 + m)) * v.npad + n) * 2 + (B & 1)] = acc[m];
      E.badj[(size_t)B * v.npad + n] = adj;
    }
  const size_t np = E.p.npad;
  for (int n = 0; n < E.p.npad; ++n) {  // the hole slots are zero
    const uint8_t dm = E.p.dmask[n];
    double u = E.p.load[n].x - E.badj[n] - E.badj[np + n];
    double w = E.p.load[n].y - E.badj[2 * np + n] - E.badj[3 * np + n];
    if (dm & 1) u = E.x[n].x;
    if (dm & 2) w = E.x[n].y;
    E.b[n] = double2{u, w};
  }
  scatter_matrix(E.p, E.A.data(), Auu, Auv, Avu, Avv);
  const size_t nvert = (size_t)(nx - 1) * (ny - 1), ncell = (size_t)nx * ny;
  std::memset(bu, 0, nvert * 8);
  std::memset(bv, 0, nvert * 8);
  scatter_vector(E.p, 0, E.b.data(), bu, bv);
  scatter_efvs(E.p, 0, E.efvs.data(), efvs);
  std::memset(eq3, 0, ncell * 4 * nl * 8);
  std::memset(omega_k, 0, ncell * (nl + 1) * 8);
  std::memset(omega, 0, ncell * 8);
  std::memset(beta_eff, 0, nvert * 8);
  for (int c = 0; c < NCELL; ++c) {
    const size_t cc = (size_t)(E.p.cell_ij[NCELL + c] - 1) * nx + (E.p.cell_ij[c] - 1);
    for (int i = 0; i < 4 * nl; ++i) eq3[cc * 4 * nl + i] = E.eq3[(size_t)c * 4 * nl + i];
    for (int k = 0; k <= nl; ++k) omega_k[cc * (nl + 1) + k] = E.omk[(size_t)c * (nl + 1) + k];
    omega[cc] = E.om[c];
  }
  for (int col = 0; col < NC; ++col) {
    const size_t w = (size_t)(E.p.col_ij[NC + col] - 1) * (nx - 1) + (E.p.col_ij[col] - 1);
    beta_eff[w] = E.beff[col];
  }
  for (int col = 0; col < NC; ++col) diva_column_velocity(E.v, col);
  scatter_velocity_3d(E.p, 0, E.x3.data(), uout, vout);
  scatter_diva(E.p, 0, E.x.data(), E.bt.data());
  return 0;
}

// The whole Picard loop of a solve (3-D, or 2-D: shallow-shelf, L1L2, DIVA)
// through the device bodies in the engine's launch order (run_picard: the sliding
// law, assembly pass 1, DIVA's omega and beta_eff, the rows and b, the
// linear solve, DIVA's traction and 3-D velocity, the Picard criterion;
// the L1L2 reconstruction after the loop), with the oracle's PCG standing
// in for the device's on the reference layout.  Outputs as bp_solve (the
// 3-D velocity, efvs; DIVA's state written back) and the Picard count.
// which_resid 0-2 only.  10 if the plan rejects the inputs.
extern "C" int emu_picard(const bp_inputs* in, const double* uvel, const double* vvel, double* uout,
                             double* vout, double* efvs, int* picard_iters) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err) || in->which_resid > 2) return 10;
  const bool d3 = !E.p.solve2d;  // the 3-D Blatter-Pattyn loop (k_asm_qp, k_asm_rows<false>)
  E.bind();
  const DevView& v = E.v;
  const HostPlan& P = E.p;
  const InstParams& ip = P.inst[0];
  const int nx = in->nx, ny = in->ny, NC = P.ncols, NCELL = P.ncells, nl = v.nl;
  const size_t nvert = (size_t)(nx - 1) * (ny - 1), np = P.npad;
  gather_velocity(P, 0, uvel, vvel, E.x.data());
  if (P.diva) gather_velocity_3d(P, 0, uvel, vvel, E.x3.data());
  RefTables T;
  fill_ref_tables(&T);
  std::vector<double2> usav(E.x);
  const size_t n3 = nvert * (size_t)v.nz;
  std::vector<double> Auu(27 * n3), Auv(27 * n3), Avu(27 * n3), Avv(27 * n3);
  std::vector<double> bu(n3), bv(n3), xu(n3), xv(n3);
  int it = 0;
  for (it = 1; it <= ip.maxiter_nonlinear; ++it) {
    usav = E.x;
    if (ip.slide.law != 0) {  // k_slide_beta, k_cell_beta
      for (int col = 0; col < NC; ++col) {
        const double2 ub = P.diva ? E.x3[(size_t)col * (nl + 1) + nl] : E.x[node_of(P, col, v.nz - 1)];
        E.p.col_beta[col] = slide_beta(ip.slide, P.col_slide[col], P.col_slide[(size_t)NC + col],
                                       P.col_slide[2 * (size_t)NC + col], ub.x, ub.y);
        if (!(E.p.col_beta[col] >= 0.0)) return 9;
      }
      for (int c = 0; c < NCELL; ++c)
        for (int q = 0; q < 4; ++q) {
          const int col = P.cell_cols[(size_t)q * NCELL + c];
          E.p.cell_beta[(size_t)q * NCELL + c] = col >= 0 ? P.col_beta[col] : 0.0;
        }
    }
    for (int e = 0; d3 && e < P.nelem; ++e) {  // k_asm_qp
      double s = 0.0;
      for (int p = 0; p < 8; ++p) {
        double out[10], eq = 0.0;
        if (!qp_element_point(v, T, e, p, out, &eq)) return 2;
        std::memcpy(&E.qp[((size_t)e * 8 + p) * 10], out, sizeof(out));
        s += eq;
      }
      E.efvs[e] = s / 8.0;
    }
    for (int c = 0; !d3 && c < NCELL; ++c) {  // k_asm2_qp
      double s = 0.0, sk[kNzMax] = {0.0};
      for (int p = 0; p < 4; ++p) {
        double out[5], eq = 0.0, ek[kNzMax];
        if (!qp2_element_point(v, T, c, p, out, &eq, ek)) return 2;
        std::memcpy(&E.qp[((size_t)c * 8 + p) * 10], out, sizeof(out));
        s += eq;
        if (P.l1l2 || P.diva)
          for (int k = 0; k < nl; ++k) sk[k] += ek[k];
      }
      if (P.l1l2 || P.diva)
        for (int k = 0; k < nl; ++k) E.efvs[(size_t)c * nl + k] = sk[k] / 4.0;
      else
        E.efvs[c] = s / 4.0;
    }
    if (P.diva) {  // k_diva_cells, k_diva_beta, k_diva_cell_beta
      for (int c = 0; c < NCELL; ++c) diva_cell_integrals(v, c);
      for (int col = 0; col < NC; ++col) diva_column_beta(v, col);
      for (int c = 0; c < NCELL; ++c)
        for (int q = 0; q < 4; ++q) {
          const int col = P.cell_cols[(size_t)q * NCELL + c];
          E.p.cell_beta[(size_t)q * NCELL + c] = col >= 0 ? E.beff[col] : 0.0;
        }
    }
    double* Ad = reinterpret_cast<double*>(E.A.data());  // k_asm_rows<true>
    for (int B = 0; B < 4; ++B)
      each_node(P, [&](size_t n, int col, int k) {
        double acc[27];
        double adj = 0.0;
        switch (B) {
          case 0: if (d3) row_assemble<0>(v, T, col, k, acc); else row_assemble2<0>(v, T, col, acc);
                  row_basal<0>(v, T, col, k, acc); adj = row_dirichlet<0>(v, col, k, acc); break;
          case 1: if (d3) row_assemble<1>(v, T, col, k, acc); else row_assemble2<1>(v, T, col, acc);
                  row_basal<1>(v, T, col, k, acc); adj = row_dirichlet<1>(v, col, k, acc); break;
          case 2: if (d3) row_assemble<2>(v, T, col, k, acc); else row_assemble2<2>(v, T, col, acc);
                  row_basal<2>(v, T, col, k, acc); adj = row_dirichlet<2>(v, col, k, acc); break;
          default: if (d3) row_assemble<3>(v, T, col, k, acc); else row_assemble2<3>(v, T, col, acc);
                   row_basal<3>(v, T, col, k, acc); adj = row_dirichlet<3>(v, col, k, acc); break;
        }
        for (int m = 0; m < 27; ++m) Ad[(((size_t)((B >> 1) * 27 + m)) * np + n) * 2 + (B & 1)] = acc[m];
        E.badj[(size_t)B * np + n] = adj;
      });
    for (int n = 0; n < (int)np; ++n) {  // k_rhs (the hole slots are zero)
      const uint8_t dm = P.dmask[n];
      double u = P.load[n].x - E.badj[n] - E.badj[np + n];
      double w = P.load[n].y - E.badj[2 * np + n] - E.badj[3 * np + n];
      if (dm & 1) u = E.x[n].x;
      if (dm & 2) w = E.x[n].y;
      E.b[n] = double2{u, w};
    }
    if (!d3 && !P.diva && ip.which_babc == 6) {  // a frozen bed: nothing is solved
      for (int n = 0; n < (int)np; ++n) E.x[n] = double2{0.0, 0.0};
    } else {  // the linear solve on the reference layout
      const int nzs = v.nz;
      scatter_matrix(P, E.A.data(), Auu.data(), Auv.data(), Avu.data(), Avv.data());
      for (double* a : {Auu.data(), Auv.data(), Avu.data(), Avv.data()}) halo_stag(nx, ny, 27 * nzs, P.periodic[0], a);
      std::fill(bu.begin(), bu.end(), 0.0);
      std::fill(bv.begin(), bv.end(), 0.0);
      std::fill(xu.begin(), xu.end(), 0.0);
      std::fill(xv.begin(), xv.end(), 0.0);
      scatter_vector(P, 0, E.b.data(), bu.data(), bv.data());
      scatter_vector(P, 0, E.x.data(), xu.data(), xv.data());
      for (double* a : {bu.data(), bv.data(), xu.data(), xv.data()}) halo_stag(nx, ny, nzs, P.periodic[0], a);
      std::vector<int> av(in->active_vertex, in->active_vertex + nvert);
      double perr = 0.0;
      int nit = 0;
      const int st = ip.variant == 3
          ? orc_pcg_chrongear_3d(nx, ny, nzs, P.periodic[0], av.data(), Auu.data(), Auv.data(), Avu.data(),
                                 Avv.data(), bu.data(), bv.data(), xu.data(), xv.data(), ip.precond,
                                 ip.pcg_maxiters, ip.pcg_tol, ip.ncheck, &perr, &nit)
          : orc_pcg_standard_3d(nx, ny, nzs, P.periodic[0], av.data(), Auu.data(), Auv.data(), Avu.data(),
                                Avv.data(), bu.data(), bv.data(), xu.data(), xv.data(), ip.precond,
                                ip.pcg_maxiters, ip.pcg_tol, ip.ncheck, &perr, &nit);
      if (st == ORC_ERR_NAN) return 1;
      for (int col = 0; col < NC; ++col) {
        const size_t w = (size_t)(P.col_ij[NC + col] - 1) * (nx - 1) + (P.col_ij[col] - 1);
        for (int k = 0; k < nzs; ++k) E.x[node_of(P, col, k)] = double2{xu[w * nzs + k], xv[w * nzs + k]};
      }
    }
    if (P.diva)  // k_diva_velocity
      for (int col = 0; col < NC; ++col) diva_column_velocity(v, col);
    double r = 0.0, rsum = 0.0;  // k_picard_check (2-D: no bed layer to leave out)
    long cnt = 0;
    const bool nobed = d3 && (ip.which_resid == 1 || ip.which_resid == 2);
    each_node(P, [&](size_t n, int, int k) {
      if (nobed && k == v.nz - 1) return;
      const double speed = std::sqrt(E.x[n].x * E.x[n].x + E.x[n].y * E.x[n].y);
      if (speed != 0.0) {
        const double old = std::sqrt(usav[n].x * usav[n].x + usav[n].y * usav[n].y);
        const double d = std::fabs((old - speed) / speed);
        r = std::max(r, d);
        rsum += d;
        ++cnt;
      }
    });
    const double crit = ip.which_resid == 2 ? (cnt > 0 ? rsum / cnt : 0.0) : r;
    if (!(crit >= 1.0e-4)) break;
  }
  *picard_iters = std::min(it, ip.maxiter_nonlinear);
  if (P.l1l2) {
    for (int c = 0; c < NCELL; ++c) l1l2_cell(v, c);
    for (int col = 0; col < NC; ++col) l1l2_column(v, col);
  }
  if (P.l1l2 || P.diva) scatter_velocity_3d(P, 0, E.x3.data(), uout, vout);
  else scatter_velocity(P, 0, E.x.data(), uout, vout);
  if (P.diva) scatter_diva(P, 0, E.x.data(), E.bt.data());
  scatter_efvs(P, 0, E.efvs.data(), efvs);
  return 0;
}

// sizeof of a C ABI struct by name (0 for an unknown name), for the
// binding's layout test.
extern "C" long emu_sizeof(const char* name) {
  const std::string n(name);
  if (n == "bp_inputs") return (long)sizeof(bp_inputs);
  if (n == "bp_stats") return (long)sizeof(bp_stats);
  if (n == "bp_model") return (long)sizeof(bp_model);
  if (n == "bp_setup_arrays") return (long)sizeof(bp_setup_arrays);
  if (n == "bp_sliding") return (long)sizeof(bp_sliding);
  if (n == "bp_l1l2") return (long)sizeof(bp_l1l2);
  if (n == "bp_diva") return (long)sizeof(bp_diva);
  return 0;
}

// gather_velocity then scatter_velocity through the host plan of one
// solve (the path of an initial guess into the device vector and of the
// solution back out).  10 if the plan rejects the inputs.
extern "C" int emu_velocity_roundtrip(const bp_inputs* in, const double* uvel, const double* vvel,
                                      double* uout, double* vout) {
  Emu E;
  std::string err;
  if (!build_plan(in, 1, &E.p, &err)) return 10;
  E.bind();
  gather_velocity(E.p, 0, uvel, vvel, E.x.data());
  scatter_velocity(E.p, 0, E.x.data(), uout, vout);
  return 0;
}
